"""End to end through the C++ model plugin and the mass-gpu driver on a GPU.

* FP64 mode on the configuration the reference wrote its golden JSON for:
  parameters.json and frame3.json must be text-identical to the reference's
  (same Configure() random stream, bit-exact steps, same JSON writer).
* Configure() of every initial configuration against the reference's.
* An FP32 run of the benchmark's initial state (random director, tanh disk)
  through several output intervals, with the runtime checks on.
"""
import json
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "mass_hd_b200", "host")
DRIVER = os.path.join(HOST, "_build", "mass-gpu")
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module", autouse=True)
def driver():
    subprocess.run(["make", "-s", "-C", HOST], check=True)
    assert os.path.exists(DRIVER)


def runcard(path, model, opts):
    lines = [f"model = {model}"] + [f"{k} = {v}" for k, v in opts.items()]
    path.write_text("\n".join(lines) + "\n")


def run(card, out, *extra):
    r = subprocess.run([DRIVER, str(card), "-o", str(out), *extra],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r


LYO = dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5, tauIso=1.5, rho=40.0,
           friction=0.0, AA=0.1, CC=0.1, LL=0.05, KK=0.05, zeta=0.01,
           zetaI=0.0, npc=1)
NEM = dict(Gamma=0.3, xi=0.7, tau=1.5, rho=40.0, friction=0.0, CC=0.1,
           LL=0.05, zeta=0.02, npc=1)


@pytest.mark.parametrize("tag", ["lyo", "nem"])
def test_fp64_output_files_identical_to_reference(tmp_path, tag):
    if tag == "lyo":
        opts = dict(LYO, config="circle", radius=2.0, level=0.0, conc=1.0, angle=0.0, noise=1.0)
        model = "lyotropic"
    else:
        opts = dict(NEM, angle=0.0, noise=1.0)
        model = "nematic"
    opts.update(LX=4, LY=3, nsteps=3, ninfo=1, seed=7, precision="fp64")
    card = tmp_path / "run.dat"
    runcard(card, model, opts)
    run(card, tmp_path / "out")
    for name, gold in (("parameters.json", f"{tag}_parameters.json"),
                       ("frame3.json", f"{tag}_frame3.json")):
        got = (tmp_path / "out" / name).read_text()
        want = open(os.path.join(GOLDEN, gold)).read()
        assert got == want, name


def test_fp64_division_output_identical_to_reference(tmp_path):
    """LyotropicWithDivision through the plugin: masks drawn on the host from
    the reference's random stream, source rate and steps on the device;
    parameters.json and frame5.json (masks included) text-identical to the
    reference's (tests/golden/gen_golden.py division)."""
    opts = dict(LYO, config="circle", radius=2.5, level=0.0, conc=1.0, angle=0.0, noise=1.0)
    opts.update({"alpha": 0.05, "beta": 0.03, "division-rate": 0.6, "division-time": 1,
                 "division-radius": 1.5, "death-rate": 0.3, "death-time": 2,
                 "death-radius": 1.0, "phi-critical": 1.5})
    opts.update(LX=8, LY=6, nsteps=5, ninfo=5, seed=7, precision="fp64")
    card = tmp_path / "run.dat"
    runcard(card, "lyotropic-with-division", opts)
    run(card, tmp_path / "out")
    for name, gold in (("parameters.json", "div_parameters.json"),
                       ("frame5.json", "div_frame5.json")):
        got = (tmp_path / "out" / name).read_text()
        want = open(os.path.join(GOLDEN, gold)).read()
        assert got == want, name


@pytest.mark.parametrize("prefix,bc,cfg,LX,LY", [("gog", 0, "noise", 16, 12),
                                                  ("gog_box", 3, "front", 12, 10)])
def test_fp64_go_or_grow_output_identical_to_reference(tmp_path, prefix, bc, cfg, LX, LY):
    """GoOrGrow through the plugin: lyotropic configuration, device
    relaxation, phenotype noise (smoothed on the host) or front, masks from
    the reference's random stream; parameters.json and frame5.json (m and
    chi included) text-identical to the reference's (tests/golden/gen_golden.py
    go-or-grow)."""
    opts = dict(LYO, config="circle", radius=3.5, level=0.0, conc=1.0, angle=0.0, noise=1.0,
                zeta=0.02)
    opts.update({"B": 0.1, "Snem": 1.0, "Dchi": 0.01, "Achi": 0.1, "Ochi": 0.05,
                 "phiswitch": 0.5, "growTogether": 1, "chi0": 0.6, "chi-noise": 0.05,
                 "chi-length": 1.5, "relax-steps": 10, "relax-dt": 1.0, "relax-phi": 1,
                 "relax-Q": 1, "alpha": 0.01, "beta": 0.005, "division-rate": 0.6,
                 "division-time": 1, "division-radius": 1.5, "death-rate": 0.3,
                 "death-time": 2, "death-radius": 1.0, "phi-critical": 0.9,
                 "chi-config": cfg})
    opts.update(LX=LX, LY=LY, bc=bc, nsteps=5, ninfo=5, seed=7, precision="fp64")
    card = tmp_path / "run.dat"
    runcard(card, "go-or-grow", opts)
    run(card, tmp_path / "out")
    for name, gold in (("parameters.json", f"{prefix}_parameters.json"),
                       ("frame5.json", f"{prefix}_frame5.json")):
        got = (tmp_path / "out" / name).read_text()
        want = open(os.path.join(GOLDEN, gold)).read()
        assert got == want, name


@pytest.mark.parametrize("nsteps", [0, 5])
def test_fp64_go_or_grow_state_bit_identical_to_reference(tmp_path, nsteps):
    """The plugin's configured state (nsteps = 0: lyotropic set-up, device
    relaxation, host phenotype noise and smoothing) and its state after 5
    steps, saved at full precision by --save-state, against the reference's
    in-memory fields bit for bit (signs of zero included)."""
    import sys
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from tests.helpers import bits_equal
    import mass_hd_b200 as M
    gog = {"B": 0.1, "Snem": 1.0, "Dchi": 0.01, "Achi": 0.1, "Ochi": 0.05,
           "phiswitch": 0.5, "growTogether": 1, "chi0": 0.6, "chi-noise": 0.05,
           "chi-length": 1.5, "relax-steps": 10, "relax-dt": 1.0, "relax-phi": 1,
           "relax-Q": 1, "alpha": 0.01, "beta": 0.005, "division-rate": 0.6,
           "division-time": 1, "division-radius": 1.5, "death-rate": 0.3,
           "death-time": 2, "death-radius": 1.0, "phi-critical": 0.9, "chi-config": "noise"}
    opts = dict(LYO, config="circle", radius=3.5, level=0.0, conc=1.0, angle=0.0, noise=1.0,
                zeta=0.02)
    opts.update(gog)
    LX, LY = 16, 12
    opts.update(LX=LX, LY=LY, nsteps=nsteps, ninfo=5, seed=7, precision="fp64")
    card = tmp_path / "run.dat"
    runcard(card, "go-or-grow", opts)
    state = tmp_path / "state.ckpt"
    run(card, tmp_path / "out", "--no-write", f"--save-state={state}")
    ref = O.RefOracle(O.GO_OR_GROW, {k: v for k, v in opts.items()
                                     if k not in ("LX", "LY", "nsteps", "ninfo", "seed",
                                                  "precision")}, LX, LY, 0)
    ref.configure(7)
    ref.step(nsteps)
    lat = M.Lattice(M.GO_OR_GROW, opts, LX, LY, 0, M.FP64)
    lat.load(str(state))
    for n in ("ff", "QQxx", "QQyx", "phi", "m", "chi"):
        assert bits_equal(lat.get(n), ref.get(n)), n
    lat.close()


def load_frame(path):
    d = json.load(open(path))["data"]
    return {k: np.asarray(v["value"], dtype=float) for k, v in d.items()}


def test_configure_matches_reference(tmp_path):
    z = np.load(os.path.join(GOLDEN, "configure.npz"))
    meta = json.loads(str(z["meta"]))
    for name, m in meta.items():
        params = dict(m["params"])
        model = "lyotropic" if m["model"] == 0 else "nematic"
        params.update(LX=m["LX"], LY=m["LY"], bc=m["bc"], nsteps=0, ninfo=1,
                      seed=m["seed"], precision="fp64")
        card = tmp_path / f"{name}.dat"
        runcard(card, model, params)
        out = tmp_path / name
        run(card, out)
        fr = load_frame(out / "frame0.json")
        for k in ("ff", "QQxx", "QQyx") + (("phi",) if model == "lyotropic" else ()):
            want = z[f"{name}__{k}"]
            got = fr[k].reshape(want.shape)
            # the frame holds 6 significant digits
            assert np.allclose(got, want, rtol=2e-6, atol=1e-6), (name, k)


def test_fp32_baseline_state_runs_with_checks(tmp_path):
    opts = dict(LYO, config="random-disk", radius=32.0, width=2.0, conc=1.0, angle=0.0,
                noise=1.0, LX=128, LY=128, nsteps=300, ninfo=100, seed=3, precision="fp32")
    card = tmp_path / "run.dat"
    runcard(card, "lyotropic", opts)
    r = run(card, tmp_path / "out")
    assert "fcheck" in r.stdout
    frames = sorted(p for p in os.listdir(tmp_path / "out") if p.startswith("frame"))
    assert frames == ["frame0.json", "frame100.json", "frame200.json", "frame300.json"]
    fr = load_frame(tmp_path / "out" / "frame300.json")
    for k in ("ff", "QQxx", "phi", "sigmaXX", "sigma_active_yx"):
        assert np.all(np.isfinite(fr[k])), k
    # phi is conserved by the flux form; mass to round-off
    f0 = load_frame(tmp_path / "out" / "frame0.json")
    assert abs(fr["phi"].sum() - f0["phi"].sum()) < 1e-2
    assert abs(fr["ff"].sum() - f0["ff"].sum()) < 1e-1


def test_step_errors_surface_in_runtime_checks(tmp_path):
    # an unknown precision is rejected at Initialize() with the model's message
    opts = dict(LYO, config="circle", radius=2, conc=1, LX=8, LY=8, nsteps=1, precision="fp16")
    card = tmp_path / "run.dat"
    runcard(card, "lyotropic", opts)
    r = subprocess.run([DRIVER, str(card), "-o", str(tmp_path / "o")], capture_output=True, text=True)
    assert r.returncode == 1 and "precision 'fp16' unknown" in r.stderr


def test_fp32_go_or_grow_driver_tracks_fp64(tmp_path):
    """mass-gpu on a go-or-grow runcard in FP32, the fused one-launch step on
    this periodic lattice (relaxation on the sweeps, masks drawn on the
    device from the reference's stream), against the same runcard in FP64:
    every frame field within FP32 tolerance after 8 steps."""
    gog = {"B": 0.1, "Snem": 1.0, "Dchi": 0.01, "Achi": 0.1, "Ochi": 0.05,
           "phiswitch": 0.5, "growTogether": 0, "chi0": 0.6, "chi-noise": 0.05,
           "chi-length": 1.5, "relax-steps": 20, "relax-dt": 1.0, "relax-phi": 1,
           "relax-Q": 1, "alpha": 0.01, "beta": 0.005, "division-rate": 0.6,
           "division-time": 1, "division-radius": 2.5, "death-rate": 0.3,
           "death-time": 2, "death-radius": 1.5, "phi-critical": 0.9, "chi-config": "noise"}
    frames = {}
    for prec in ("fp32", "fp64"):
        opts = dict(LYO, config="circle", radius=20, level=0.0, conc=1.0, angle=0.0, noise=1.0,
                    zeta=0.02)
        opts.update(gog)
        opts.update(LX=64, LY=64, nsteps=8, ninfo=8, seed=11, precision=prec)
        card = tmp_path / f"{prec}.dat"
        runcard(card, "go-or-grow", opts)
        run(card, tmp_path / prec)
        frames[prec] = load_frame(tmp_path / prec / "frame8.json")
    a, b = frames["fp32"], frames["fp64"]
    for k in ("QQxx", "QQyx", "phi", "m", "chi", "division_mask", "death_mask"):
        assert k in a, k
    for k in ("division_mask", "death_mask"):
        assert np.array_equal(a[k], b[k]), k
    rest = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4) * 40.0
    for k in ("ff", "QQxx", "QQyx", "phi", "m"):
        x, y = a[k], b[k]
        if k == "ff":
            x, y = x.reshape(-1, 9) - rest, y.reshape(-1, 9) - rest
        assert np.linalg.norm(x - y) <= 1e-4 * np.linalg.norm(y), k
