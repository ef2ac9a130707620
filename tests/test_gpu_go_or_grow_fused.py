"""Go-or-grow in the fused FP32 warp-strip kernel (one launch per step).

Periodic FP32 go-or-grow lattices with npc = 1, LY a multiple of 4 and at
least 64 run the whole step - the lyotropic update, the phenotype density m
with its chi-weighted fluxes, phenotype diffusion, switching potential and
growth, the clamp of m and the division/death source - in one launch of the
fused kernel, with chi = m/phi formed on the fly. Checked against the FP64
mode (bit-identical to the reference's GoOrGrow) started from the
reference's own Configure() state and fed the reference's masks step by
step: state fields, chi and the derived fields within FP32 tolerances, both
growth rules. Also: tile invariance, the dry relaxation and conserve_phi
(both run on the unfused sweeps and the lattice carries on), checkpoints.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import bits_equal, ff_dev, rel_l2
from tests.test_gpu_go_or_grow import DERIVED, STATE, params, rate_of

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402


def pair_run(p, LX, LY, steps, seed=3):
    ref = O.RefOracle(O.GO_OR_GROW, p, LX, LY, 0)
    ref.configure(seed)
    st = {n: ref.get(n) for n in STATE}
    a = M.Lattice(M.GO_OR_GROW, p, LX, LY, 0, M.FP32)
    b = M.Lattice(M.GO_OR_GROW, p, LX, LY, 0, M.FP64)
    assert a.uses_fused and a.launches_per_step == 1
    a.upload_state(st)
    b.upload_state(st)
    masked = 0
    for _ in range(steps):
        ref.step(1)
        rate, k = rate_of(ref, p)
        masked += k
        a.set_phi_source(rate)
        b.set_phi_source(rate)
        a.step(1)
        b.step(1)
    return a, b, masked


@pytest.mark.parametrize("grow", [0, 1])
def test_fused_go_or_grow_within_fp32_tolerance(grow):
    a, b, masked = pair_run(params(growTogether=grow), 64, 128, 20)
    assert masked > 0
    for n in STATE + ("chi",):
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x, 40.0), ff_dev(y, 40.0)
        assert rel_l2(x, y) < 1e-4, n
    # the derived fields of the last step (the fused kernel replays it)
    for n in DERIVED:
        if n == "chi":
            continue
        x, y = a.get(n), b.get(n)
        if n == "n":
            x, y = x - 40.0, y - 40.0
        assert rel_l2(x, y) < 1e-3, n
    a.close()
    b.close()


def test_fused_go_or_grow_tiles_bit_identical():
    p = params()
    ref = O.RefOracle(O.GO_OR_GROW, p, 72, 128, 0)
    ref.configure(6)
    st = {n: ref.get(n) for n in STATE}
    rate = np.where(st["phi"] > 0.5, 0.002, 0.0)
    out = []
    for rows in (16, 64):
        lat = M.Lattice(M.GO_OR_GROW, p, 72, 128, 0, M.FP32)
        lat.set_tile(32, rows)
        lat.upload_state(st)
        lat.set_phi_source(rate)
        lat.step(9)
        out.append({n: lat.get(n) for n in STATE})
        lat.close()
    for n in STATE:
        assert bits_equal(out[0][n], out[1][n]), n


def test_fused_go_or_grow_relaxation_then_conserve_phi():
    """The dry relaxation of a fused lattice runs on the sweeps' state and
    comes back; switching conserve_phi on hands the lattice to the sweeps
    for good. Both track the FP64 mode."""
    p = params(alpha=0.0, beta=0.0)
    LX, LY = 64, 96
    ref = O.RefOracle(O.GO_OR_GROW, params(**{"relax-steps": 0}), LX, LY, 0)
    ref.configure(4)
    st = {n: ref.get(n) for n in ("ff", "QQxx", "QQyx", "phi", "m")}
    a = M.Lattice(M.GO_OR_GROW, p, LX, LY, 0, M.FP32)
    b = M.Lattice(M.GO_OR_GROW, p, LX, LY, 0, M.FP64)
    for lat in (a, b):
        lat.upload_state(st)
    ta = a.relax_free_energy(20, 0.8, True, True)
    tb = b.relax_free_energy(20, 0.8, True, True)
    assert a.uses_fused
    assert ta == pytest.approx(tb, rel=1e-5)
    for n in ("QQxx", "QQyx", "phi"):
        assert rel_l2(a.get(n), b.get(n)) < 1e-5, n
    for lat in (a, b):
        lat.set_phi_conservation(True, tb)
    assert not a.uses_fused
    a.step(30)
    b.step(30)
    assert abs(a.get("phi").sum() - tb) < 1e-4 * tb
    for n in ("phi", "m", "QQxx"):
        assert rel_l2(a.get(n), b.get(n)) < 1e-4, n
    a.close()
    b.close()


def test_fused_go_or_grow_checkpoint_and_m_upload(tmp_path):
    p = params()
    ref = O.RefOracle(O.GO_OR_GROW, p, 64, 64, 0)
    ref.configure(2)
    st = {n: ref.get(n) for n in STATE}
    rate = np.where(st["phi"] > 0.5, 0.002, 0.0)
    a = M.Lattice(M.GO_OR_GROW, p, 64, 64, 0, M.FP32)
    assert a.uses_fused
    a.upload_state(st)
    # m and chi come back as uploaded (FP32 values)
    assert rel_l2(a.get("m"), st["m"]) < 1e-7
    phi = a.get("phi")
    chi = np.where(phi > 1e-12, a.get("m") / np.where(phi > 1e-12, phi, 1.0), 0.0)
    assert np.allclose(a.get("chi"), chi, rtol=1e-6, atol=1e-7)
    a.set_phi_source(rate)
    a.step(4)
    path = os.path.join(tmp_path, "gog32.ckpt")
    a.save(path)
    a.step(4)
    b = M.Lattice(M.GO_OR_GROW, p, 64, 64, 0, M.FP32)
    b.load(path)
    b.set_phi_source(rate)
    b.step(4)
    for n in STATE:
        assert bits_equal(a.get(n), b.get(n)), n
    # a cleared source is a zero growth rate
    a.set_phi_source(None)
    b.set_phi_source(np.zeros(64 * 64))
    a.step(2)
    b.step(2)
    for n in STATE:
        assert bits_equal(a.get(n), b.get(n)), n
    a.close()
    b.close()
