"""FP32 production mode against the FP64 oracle mode (same GPU, same input).

Tolerances (relative L2 per field; populations compared as deviations
f_v - t_v*rho so the rest state cannot hide errors):
  * 1 step:   <= 2e-5 on every state field
  * 10 steps: <= 1e-4
These are the FP32 rounding of the step arithmetic; the measured per-field
errors are printed with -s. Long runs diverge chaotically and are compared
statistically (tests/test_gpu_stats.py).

Also checked: every tile shape of the fused kernel gives bit-identical
results (each site's arithmetic does not depend on the tiling), ragged
lattices, the diagnostic-field replay, and the unfused FP32 wall path.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_ALL, LYO_C1, NEM_ALL, NEM_C2, ff_dev, rel_l2

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402

STATE_FIELDS = {O.LYOTROPIC: ("ff", "QQxx", "QQyx", "phi"), O.NEMATIC: ("ff", "QQxx", "QQyx")}


def errors(a, b, model, rho=40.0):
    out = {}
    for n in STATE_FIELDS[model]:
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x, rho), ff_dev(y, rho)
        out[n] = rel_l2(x, y)
    return out


def pair(model, params, LX, LY, bc, st):
    a = M.Lattice(model, params, LX, LY, bc, M.FP32)
    b = M.Lattice(model, params, LX, LY, bc, M.FP64)
    a.upload_state(st)
    b.upload_state(st)
    return a, b


@pytest.mark.parametrize("model,params", [(O.LYOTROPIC, LYO_C1), (O.LYOTROPIC, LYO_ALL),
                                          (O.NEMATIC, NEM_C2), (O.NEMATIC, NEM_ALL)])
def test_fp32_fused_vs_fp64(model, params):
    LX, LY = 96, 256
    st = O.synthetic_state(model, LX, LY, seed=21, flow=0.01)
    a, b = pair(model, params, LX, LY, 0, st)
    assert a.uses_fused
    a.step(1)
    b.step(1)
    e1 = errors(a, b, model)
    a.step(9)
    b.step(9)
    e10 = errors(a, b, model)
    print("fp32 vs fp64", model, "1 step", e1, "10 steps", e10)
    for n, e in e1.items():
        assert e <= 2e-5, (n, e)
    for n, e in e10.items():
        assert e <= 1e-4, (n, e)


def test_fp32_matches_reference_golden_loosely():
    from tests.helpers import golden_cases, load_golden
    for path in golden_cases():
        meta, z = load_golden(path)
        if meta["bc"] not in (0, 1, 2, 3, 4) or meta["LY"] < 4:
            continue
        L = M.Lattice(meta["model"], meta["params"], meta["LX"], meta["LY"], meta["bc"], M.FP32)
        L.upload(z["in_ff"], z["in_QQxx"], z["in_QQyx"], z["in_phi"] if "in_phi" in z.files else None)
        L.step(meta["steps"])
        assert rel_l2(ff_dev(L.get("ff")), ff_dev(z["out_ff"])) < 1e-4, path
        assert rel_l2(L.get("QQxx"), z["out_QQxx"]) < 1e-4, path


@pytest.mark.parametrize("model", [O.LYOTROPIC, O.NEMATIC])
def test_fused_tiles_bit_identical(model):
    params = LYO_ALL if model == O.LYOTROPIC else NEM_ALL
    LX, LY = 70, 264           # ragged: 264 = 4*56 + 40 (NT=64), partial chunks
    st = O.synthetic_state(model, LX, LY, seed=4, flow=0.01)
    ref = None
    for nt, rows in ((64, 16), (64, 70), (128, 32), (128, 13), (256, 64), (256, 1)):
        L = M.Lattice(model, params, LX, LY, 0, M.FP32)
        L.set_tile(nt, rows)
        L.upload_state(st)
        L.step(3)
        got = {n: L.get(n) for n in STATE_FIELDS[model]}
        if ref is None:
            ref = got
        else:
            for n in got:
                assert np.array_equal(got[n], ref[n]), (nt, rows, n)


@pytest.mark.parametrize("model", [O.LYOTROPIC, O.NEMATIC])
def test_warp_strip_tiles_bit_identical_and_close_to_fp64(model):
    # the warp-strip kernel (packed FP32x2) rounds differently from the
    # CTA-strip kernel, so it is compared with itself across tiles and with
    # the FP64 mode within the FP32 tolerance
    params = LYO_ALL if model == O.LYOTROPIC else NEM_ALL
    LX, LY = 70, 264
    st = O.synthetic_state(model, LX, LY, seed=5, flow=0.01)
    ref = None
    for rows in (16, 70, 9, 1):
        L = M.Lattice(model, params, LX, LY, 0, M.FP32)
        L.set_tile(32, rows)
        L.upload_state(st)
        L.step(3)
        got = {n: L.get(n) for n in STATE_FIELDS[model]}
        if ref is None:
            ref = got
        else:
            for n in got:
                assert np.array_equal(got[n], ref[n]), (rows, n)
    b = M.Lattice(model, params, LX, LY, 0, M.FP64)
    b.upload_state(st)
    b.step(3)
    for n in STATE_FIELDS[model]:
        x, y = ref[n], b.get(n)
        if n == "ff":
            x, y = ff_dev(x), ff_dev(y)
        assert rel_l2(x, y) <= 5e-5, (n, rel_l2(x, y))


def test_fused_autotune_picks_a_valid_tile():
    L = M.Lattice(O.LYOTROPIC, LYO_C1, 256, 256, 0, M.FP32)
    st = O.synthetic_state(O.LYOTROPIC, 256, 256, seed=1)
    L.upload_state(st)
    L.autotune()
    nt, rows = L.tile()
    assert nt in (32, 64, 128, 256) and rows >= 1
    before = L.get("ff")
    assert np.array_equal(before, L.get("ff"))   # tuning does not advance the state
    L.step(2)


def test_fp32_diagnostic_replay_matches_fp64():
    LX, LY = 64, 128
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=9, flow=0.01)
    a, b = pair(O.LYOTROPIC, LYO_ALL, LX, LY, 0, st)
    with pytest.raises(M.MassLBError):
        a.get("sigmaXX")      # no step yet
    a.step(3)
    b.step(3)
    ff_before = a.get("ff")
    for n in ("n", "ux", "uy", "ux_phi", "uy_phi", "HHxx", "HHyx", "MU", "dxQQxx",
              "dyQQyx", "sigmaXX", "sigmaYY", "sigmaXY", "sigmaYX", "sigma_bulk",
              "sigma_elastic_xx", "sigma_elastic_yx", "sigma_phase_field_xx",
              "sigma_phase_field_yx", "sigma_active_xx", "sigma_active_yx"):
        x, y = a.get(n), b.get(n)
        if n == "n":
            x, y = x - 40.0, y - 40.0
        scale = max(np.abs(y).max(), 1e-12)
        assert np.max(np.abs(x - y)) <= 1e-4 * scale + 1e-7, n
    # the replay leaves the state bit-identical
    assert np.array_equal(ff_before, a.get("ff"))
    a.step(1)
    b.step(1)
    assert rel_l2(ff_dev(a.get("ff")), ff_dev(b.get("ff"))) < 1e-4


@pytest.mark.parametrize("bc", [1, 2, 3, 4])
def test_fp32_walls_vs_fp64(bc):
    LX, LY = 40, 36
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=30 + bc, flow=0.01)
    a, b = pair(O.LYOTROPIC, LYO_ALL, LX, LY, bc, st)
    assert not a.uses_fused
    a.step(10)
    b.step(10)
    for n, e in errors(a, b, O.LYOTROPIC).items():
        assert e <= 1e-4, (bc, n, e)


def test_fp32_unfused_when_not_fusable():
    # LY not a multiple of 4 -> unfused FP32 kernels, still correct
    LX, LY = 30, 66
    st = O.synthetic_state(O.NEMATIC, LX, LY, seed=2, flow=0.01)
    a, b = pair(O.NEMATIC, NEM_ALL, LX, LY, 0, st)
    assert not a.uses_fused
    a.step(5)
    b.step(5)
    for n, e in errors(a, b, O.NEMATIC).items():
        assert e <= 1e-4, (n, e)


def test_fp32_conservation():
    LX, LY = 128, 128
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=12, flow=0.01)
    L = M.Lattice(O.LYOTROPIC, LYO_C1, LX, LY, 0, M.FP32)
    L.upload_state(st)
    ftot, ptot = L.initial_totals()
    L.step(200)
    f, p = L.runtime_checks()
    assert abs(f - ftot) < 1e-6 * ftot
    assert abs(p - ptot) < 1e-4 * LX * LY * 1e-3 + 1e-3
