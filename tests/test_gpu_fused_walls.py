"""FP32 fused step on lattices with walls (bc 1-4 lyotropic and go-or-grow,
bc 1 nematic): the warp-strip kernel over the whole lattice plus the wall
bands (the 8 rows next to each wall, stepped by the wall-aware sweeps, of
which the outer 4 are kept).

Checked here:
  * against the FP64 mode (bit-identical to the reference's build) with the
    FP32 tolerances of tests/test_gpu_fp32.py: relative L2 <= 1e-4 per state
    field after 10 steps; derived fields within 1e-4 of their scale;
  * the interior: after one step, every site at least 4 sites from a wall
    equals the periodic fused step of the same state bit for bit, and the
    band rows differ from it (the walls act there);
  * a division source, go-or-grow without phi conservation, the hand-over
    to the sweeps when conservation is switched on (the ghost-ring aware
    copy of the state), and a checkpoint round trip.
The decomposition itself is pinned in FP64 on the CPU by
tests/test_wall_bands.py.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_ALL, NEM_ALL, bits_equal, ff_dev, rel_l2

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402

STATE = {O.LYOTROPIC: ("ff", "QQxx", "QQyx", "phi"), O.NEMATIC: ("ff", "QQxx", "QQyx"),
         O.GO_OR_GROW: ("ff", "QQxx", "QQyx", "phi", "m")}
DERIVED = ("n", "ux", "uy", "HHxx", "HHyx", "dxQQxx", "dyQQxx", "dxQQyx", "dyQQyx",
           "sigmaXX", "sigmaYY", "sigmaYX", "sigmaXY")
DERIVED_LYO = ("ux_phi", "uy_phi", "MU", "sigma_bulk", "sigma_elastic_xx", "sigma_elastic_yx",
               "sigma_phase_field_xx", "sigma_phase_field_yx", "sigma_active_xx",
               "sigma_active_yx")
CASES = [(O.LYOTROPIC, LYO_ALL, bc) for bc in (1, 2, 3, 4)] + [(O.NEMATIC, NEM_ALL, 1)]
# two correctors: the bands keep 6 rows of 12-row halves
CASES_NPC2 = [(O.LYOTROPIC, dict(LYO_ALL, npc=2), 1), (O.LYOTROPIC, dict(LYO_ALL, npc=2), 4),
              (O.NEMATIC, dict(NEM_ALL, npc=2), 1)]


def errors(a, b, model, rho=40.0):
    out = {}
    for n in STATE[model]:
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


@pytest.mark.parametrize("model,params,bc", CASES + CASES_NPC2)
def test_fused_walls_vs_fp64(model, params, bc):
    LX, LY = 72, 96
    st = O.synthetic_state(model, LX, LY, seed=50 + bc, flow=0.01)
    a, b = pair(model, params, LX, LY, bc, st)
    assert a.uses_fused and a.launches_per_step > 1
    a.step(10)
    b.step(10)
    for n, e in errors(a, b, model).items():
        assert e <= 1e-4, (bc, n, e)
    names = DERIVED + (DERIVED_LYO if model == O.LYOTROPIC else ())
    for n in names:
        x, y = a.get(n), b.get(n)
        if n == "n":
            x, y = x - 40.0, y - 40.0
        scale = max(np.abs(y).max(), 1e-12)
        assert np.max(np.abs(x - y)) <= 1e-4 * scale + 1e-7, (bc, n)


@pytest.mark.parametrize("model,params,bc", CASES + CASES_NPC2)
def test_fused_walls_interior_is_the_periodic_step(model, params, bc):
    LX, LY = 40, 64
    st = O.synthetic_state(model, LX, LY, seed=70 + bc, flow=0.02)
    w = M.Lattice(model, params, LX, LY, bc, M.FP32)
    p = M.Lattice(model, params, LX, LY, 0, M.FP32)
    assert w.uses_fused and p.uses_fused
    w.upload_state(st)
    p.upload_state(st)
    w.step(1)
    p.step(1)
    box = model != O.NEMATIC and bc in (3, 4)
    k = 2 + 2 * params.get("npc", 1)     # rows one step reaches
    inner = np.zeros((LX, LY), dtype=bool)
    inner[k if box else 0:LX - k if box else LX, k:LY - k] = True
    for n in STATE[model]:
        x = w.get(n).reshape(LX, LY, -1)
        y = p.get(n).reshape(LX, LY, -1)
        assert bits_equal(x[inner], y[inner]), n
    # the walls act on the band rows
    fw = w.get("ff").reshape(LX, LY, 9)
    fp = p.get("ff").reshape(LX, LY, 9)
    assert not np.array_equal(fw[:, :k], fp[:, :k])
    assert not np.array_equal(fw[:, LY - k:], fp[:, LY - k:])
    if box:
        assert not np.array_equal(fw[:k], fp[:k])


@pytest.mark.parametrize("bc", [2, 3])
def test_fused_walls_with_division_source(bc):
    LX, LY = 64, 96
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=90 + bc, flow=0.01)
    a, b = pair(O.LYOTROPIC, LYO_ALL, LX, LY, bc, st)
    assert a.uses_fused
    rate = np.random.default_rng(bc).uniform(-2e-3, 4e-3, LX * LY)
    a.set_phi_source(rate)
    b.set_phi_source(rate)
    a.step(10)
    b.step(10)
    for n, e in errors(a, b, O.LYOTROPIC).items():
        assert e <= 1e-4, (bc, n, e)


@pytest.mark.parametrize("bc", [1, 4])
def test_fused_walls_go_or_grow(bc):
    """Go-or-grow with walls and without phi conservation (with it, the
    global phi sum enters every site and the lattice runs the sweeps),
    masks of the reference's own model fed step by step."""
    from tests.test_gpu_go_or_grow import params, rate_of
    p = params()
    LX, LY = 64, 96
    ref = O.RefOracle(O.GO_OR_GROW, p, LX, LY, bc)
    ref.configure(3)
    st = {n: ref.get(n) for n in STATE[O.GO_OR_GROW]}
    a = M.Lattice(M.GO_OR_GROW, p, LX, LY, bc, M.FP32)
    b = M.Lattice(M.GO_OR_GROW, p, LX, LY, bc, M.FP64)
    assert a.uses_fused
    a.upload_state(st)
    b.upload_state(st)
    for _ in range(10):
        ref.step(1)
        rate, _ = rate_of(ref, p)
        a.set_phi_source(rate)
        b.set_phi_source(rate)
        a.step(1)
        b.step(1)
    for n in STATE[O.GO_OR_GROW] + ("chi",):
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x, 40.0), ff_dev(y, 40.0)
        assert rel_l2(x, y) < 1e-4, (bc, n)


def test_fused_walls_hand_over_to_the_sweeps():
    """Switching phi conservation on moves a fused walled lattice to the
    sweeps (the state copied into the ghost-ring layout); it carries on
    like the FP64 mode."""
    LX, LY, bc = 64, 96, 4
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=11, flow=0.01)
    a, b = pair(O.LYOTROPIC, LYO_ALL, LX, LY, bc, st)
    a.step(3)
    b.step(3)
    assert a.uses_fused
    total = float(np.sum(b.get("phi")))
    a.set_phi_conservation(True, total)
    b.set_phi_conservation(True, total)
    assert not a.uses_fused
    a.step(7)
    b.step(7)
    for n, e in errors(a, b, O.LYOTROPIC).items():
        assert e <= 1e-4, (n, e)


def test_fused_walls_checkpoint_round_trip(tmp_path):
    LX, LY, bc = 64, 96, 1
    st = O.synthetic_state(O.NEMATIC, LX, LY, seed=12, flow=0.01)
    a = M.Lattice(O.NEMATIC, NEM_ALL, LX, LY, bc, M.FP32)
    a.upload_state(st)
    a.step(4)
    path = os.path.join(str(tmp_path), "walls.ckpt")
    a.save(path)
    a.step(5)
    b = M.Lattice(O.NEMATIC, NEM_ALL, LX, LY, bc, M.FP32)
    b.load(path)
    b.step(5)
    for n in STATE[O.NEMATIC]:
        assert bits_equal(a.get(n), b.get(n)), n


@pytest.mark.parametrize("bc", [2, 3])
def test_fused_walls_go_or_grow_relaxation(bc):
    """Go-or-grow's dry relaxation runs on the sweeps' state: a walled fused
    lattice goes there through the ghost-ring layout and comes back, then
    steps on, tracking the FP64 mode."""
    from tests.test_gpu_go_or_grow import params
    p = params(alpha=0.0, beta=0.0)
    LX, LY = 64, 96
    ref = O.RefOracle(O.GO_OR_GROW, params(**{"relax-steps": 0}), LX, LY, bc)
    ref.configure(4)
    st = {n: ref.get(n) for n in STATE[O.GO_OR_GROW]}
    a = M.Lattice(M.GO_OR_GROW, p, LX, LY, bc, M.FP32)
    b = M.Lattice(M.GO_OR_GROW, p, LX, LY, bc, M.FP64)
    for lat in (a, b):
        lat.upload_state(st)
    ta = a.relax_free_energy(20, 0.8, True, True)
    tb = b.relax_free_energy(20, 0.8, True, True)
    assert a.uses_fused
    assert ta == pytest.approx(tb, rel=1e-5)
    for n in ("QQxx", "QQyx", "phi"):
        assert rel_l2(a.get(n), b.get(n)) < 1e-5, n
    a.step(10)
    b.step(10)
    for n in STATE[O.GO_OR_GROW]:
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x, 40.0), ff_dev(y, 40.0)
        assert rel_l2(x, y) < 1e-4, n
