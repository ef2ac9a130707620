"""The CPU oracle restatement against the reference's own outputs.

Golden fixtures were produced by the reference's model sources themselves
(tests/golden/gen_golden.py); the restatement must agree bit for bit.
When the reference library (oracle/_ref) is present it is also compared
live on fresh seeded states.
"""
import glob
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "*_bc*.npz")))


def load_case(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    return meta, z


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_port_matches_reference_golden(path):
    meta, z = load_case(path)
    P = O.PortOracle(meta["model"], meta["params"], meta["LX"], meta["LY"], meta["bc"])
    for k in z.files:
        if k.startswith("in_"):
            P.set(k[3:], z[k])
    P.step(meta["steps"])
    for k in z.files:
        if k.startswith("out_"):
            got, want = P.get(k[4:]), z[k]
            assert np.array_equal(got, want), (k, np.max(np.abs(got - want)))


def test_golden_cases_cover_models_and_walls():
    metas = [load_case(p)[0] for p in CASES]
    assert {m["model"] for m in metas} == {O.LYOTROPIC, O.NEMATIC}
    assert {m["bc"] for m in metas if m["model"] == O.LYOTROPIC} >= {0, 1, 2, 3, 4, 5}
    assert any(m["params"].get("npc", 1) > 1 for m in metas)


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")

LYO = dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5, tauIso=1.3, rho=40.0,
           friction=0.02, AA=0.1, CC=0.1, LL=0.05, KK=0.05, zeta=0.03,
           zetaI=0.01, conc=0.9, npc=1)
NEM = dict(Gamma=0.3, xi=0.7, tau=1.5, rho=40.0, friction=0.01, CC=0.1,
           LL=0.05, zeta=0.02, npc=1)


@needs_ref
@pytest.mark.parametrize("model,bc", [(O.LYOTROPIC, b) for b in range(6)] + [(O.NEMATIC, b) for b in (0, 1, 2)])
def test_port_matches_reference_live(model, bc):
    params = LYO if model == O.LYOTROPIC else NEM
    LX, LY = 11, 14
    st = O.synthetic_state(model, LX, LY, seed=100 + bc, flow=0.02, phi_kind="noise")
    P = O.PortOracle(model, params, LX, LY, bc)
    R = O.RefOracle(model, params, LX, LY, bc)
    for k, v in st.items():
        P.set(k, v)
        R.set(k, v)
    P.step(6)
    R.step(6)
    names = ("ff", "fn") + (O.SCALAR_FIELDS_LYO if model == O.LYOTROPIC else O.SCALAR_FIELDS_NEM)
    for n in names:
        assert np.array_equal(P.get(n), R.get(n)), n


def test_port_conserves_mass():
    LX, LY = 16, 16
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=5, flow=0.01)
    P = O.PortOracle(O.LYOTROPIC, LYO, LX, LY, 0)
    for k, v in st.items():
        P.set(k, v)
    f0, p0 = P.totals()
    P.step(20)
    f1, p1 = P.totals()
    assert abs(f1 - f0) < 1e-8 * f0
    assert abs(p1 - p0) < 1e-9 * LX * LY


@needs_ref
def test_reference_go_or_grow_reproduces_golden_json(tmp_path):
    """The reference build's GoOrGrow (configure with relaxation and
    phenotype set-up, 5 steps with division and death) writes exactly the
    committed fixtures, which the GPU plugin test compares against."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gen_golden", os.path.join(os.path.dirname(__file__), "golden", "gen_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    gen.gen_json_gog(str(tmp_path))
    for prefix, *_ in gen.GOG_CASES:
        for part in ("parameters", "frame5"):
            name = f"{prefix}_{part}.json"
            got = (tmp_path / name).read_text()
            want = open(os.path.join(os.path.dirname(__file__), "golden", name)).read()
            assert got == want, name
    frame = json.loads(open(os.path.join(os.path.dirname(__file__), "golden",
                                         "gog_frame5.json")).read())["data"]
    assert {"m", "chi", "division_mask", "death_mask"} <= set(frame)
