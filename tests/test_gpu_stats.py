"""mass_lb_statistics on the GPU: the reference's post-processing estimators
(defect counts, <|u|^2>, enstrophy, phi-interface length) on the device,
against values produced by the reference's own Python code; and FP32 vs
FP64 agreement of window-averaged statistics in active turbulence."""
import glob
import json
import os

import numpy as np
import pytest

from oracle import stats as S

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402
from mass_hd_b200 import compare_precision as CP  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "stats_*.npz")))


def load(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    return meta, {k: z[k] for k in z.files if k != "meta"}


@pytest.mark.parametrize("precision", [M.FP64, M.FP32])
@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_statistics_match_reference_post(path, precision):
    meta, st = load(path)
    L = M.Lattice(meta["model"], meta["params"], meta["LX"], meta["LY"], 0, precision)
    if precision == M.FP32 and meta["LY"] % 4:
        pytest.skip("fused layout needs LY % 4 == 0")
    L.upload_state(st)
    got = L.statistics()
    want = meta["stats"]
    rel = 1e-10 if precision == M.FP64 else 2e-5
    assert got["defects_plus"] == want["defects_plus"]
    assert got["defects_minus"] == want["defects_minus"]
    assert got["mean_u2"] == pytest.approx(want["mean_u2"], rel=rel)
    assert got["enstrophy_density"] == pytest.approx(want["enstrophy_density"], rel=rel)
    if "perimeter" in want:
        assert got["perimeter"] == want["perimeter"]
        assert got["enstrophy_density_phi"] == pytest.approx(want["enstrophy_density_phi"], rel=rel)


def test_statistics_match_restatement_on_walls():
    # FP64 on a wall lattice: the estimators see the domain, periodically
    meta, st = load(CASES[0])
    from oracle import oracle as O
    LX, LY = 40, 36
    s = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=9, flow=0.01)
    params = dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5, tauIso=1.5, rho=40.0,
                  AA=0.1, CC=0.1, LL=0.05, KK=0.05, zeta=0.03, conc=1.0, npc=1)
    L = M.Lattice(O.LYOTROPIC, params, LX, LY, 3, M.FP64)
    L.upload_state(s)
    L.step(20)
    state = {k: L.get(k) for k in ("ff", "QQxx", "QQyx", "phi")}
    want = S.statistics(state, LX, LY)
    got = L.statistics()
    for k in ("defects_plus", "defects_minus", "perimeter"):
        assert got[k] == want[k], k
    for k in ("mean_u2", "enstrophy_density", "enstrophy_density_phi"):
        assert got[k] == pytest.approx(want[k], rel=1e-10), k


def test_fp32_vs_fp64_window_statistics_active_turbulence():
    r = CP.compare("nematic", 512, field_steps=100, steps=2500, window=1000, every=50)
    print(json.dumps(r))
    for n, e in r["field_rel_l2"].items():
        assert e < 1e-3, (n, e)
    for k in ("defect_density", "mean_u2", "enstrophy_density"):
        assert r["window"]["means"][k]["rel_diff"] < 0.05, (k, r["window"]["means"][k])
