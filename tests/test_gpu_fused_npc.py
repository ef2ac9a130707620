"""FP32 fused step with npc > 1 correctors (lyotropic and nematic, periodic).

The warp-strip kernel runs the predictor and the first corrector and also
writes the step's predictor values (the moved fn and QN of every site); each
further corrector is the sweeps' corrector sub-step on a view of the fused
planes. Checked against the FP64 mode (bit-identical to the reference's
build): the state after 10 steps within the FP32 tolerance of
tests/test_gpu_fp32.py (relative L2 <= 1e-4), the derived fields of the last
corrector within 1e-4 of their scale, with a division source too; the
launch count; and that a tile of the CTA-strip kernel is refused.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_ALL, NEM_ALL, ff_dev, rel_l2

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402

STATE = {O.LYOTROPIC: ("ff", "QQxx", "QQyx", "phi"), O.NEMATIC: ("ff", "QQxx", "QQyx")}
DERIVED = ("n", "ux", "uy", "HHxx", "HHyx", "dxQQxx", "dyQQxx", "dxQQyx", "dyQQyx",
           "sigmaXX", "sigmaYY", "sigmaYX", "sigmaXY")
DERIVED_LYO = ("ux_phi", "uy_phi", "MU", "sigma_bulk", "sigma_elastic_xx", "sigma_elastic_yx",
               "sigma_phase_field_xx", "sigma_phase_field_yx", "sigma_active_xx",
               "sigma_active_yx")


def pair(model, params, LX, LY, st):
    a = M.Lattice(model, params, LX, LY, 0, M.FP32)
    b = M.Lattice(model, params, LX, LY, 0, M.FP64)
    a.upload_state(st)
    b.upload_state(st)
    return a, b


def check_state(a, b, model, tol=1e-4):
    for n in STATE[model]:
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x, 40.0), ff_dev(y, 40.0)
        assert rel_l2(x, y) <= tol, n


@pytest.mark.parametrize("model,params,npc", [(O.LYOTROPIC, LYO_ALL, 2), (O.LYOTROPIC, LYO_ALL, 3),
                                              (O.NEMATIC, NEM_ALL, 2)])
def test_fused_npc_vs_fp64(model, params, npc):
    LX, LY = 64, 128
    p = dict(params, npc=npc)
    st = O.synthetic_state(model, LX, LY, seed=60 + npc, flow=0.01)
    a, b = pair(model, p, LX, LY, st)
    assert a.uses_fused and a.launches_per_step == npc
    a.step(10)
    b.step(10)
    check_state(a, b, model)
    names = DERIVED + (DERIVED_LYO if model == O.LYOTROPIC else ())
    for n in names:
        x, y = a.get(n), b.get(n)
        if n == "n":
            x, y = x - 40.0, y - 40.0
        scale = max(np.abs(y).max(), 1e-12)
        assert np.max(np.abs(x - y)) <= 1e-4 * scale + 1e-7, n


def test_fused_npc_with_division_source():
    LX, LY = 64, 128
    p = dict(LYO_ALL, npc=2)
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=77, flow=0.01)
    a, b = pair(O.LYOTROPIC, p, LX, LY, st)
    rate = np.random.default_rng(5).uniform(-2e-3, 4e-3, LX * LY)
    a.set_phi_source(rate)
    b.set_phi_source(rate)
    a.step(10)
    b.step(10)
    check_state(a, b, O.LYOTROPIC)


def test_fused_npc_refuses_cta_strip_tiles():
    a = M.Lattice(O.LYOTROPIC, dict(LYO_ALL, npc=2), 64, 128, 0, M.FP32)
    with pytest.raises(M.MassLBError):
        a.set_tile(64, 32)
    a.set_tile(32, 32)
