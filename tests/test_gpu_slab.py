"""x-slab decomposition on the GPU (mass_lb_get_rows / put_rows /
checks_rows and mass_hd_b200/slab.py).

One GPU runs several slabs of one lattice, the ranks emulated in one
process (halo rows moved by device copies): after every step the owned
rows must equal the whole lattice stepped on its own, bit for bit, in the
FP64 mode, the FP32 fused kernel and the FP32 unfused sweeps, and the
conservation sums over the slabs must equal the whole lattice's. A single
rank through the distributed exchange (its halos are its own periodic
images) must match too. The multi-process exchange itself is covered on
the CPU by tests/test_slab_dist.py.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_ALL, NEM_ALL, bits_equal

pytestmark = pytest.mark.gpu

import torch  # noqa: E402

import mass_hd_b200 as M  # noqa: E402
from mass_hd_b200 import slab as S  # noqa: E402

FIELDS = {M.LYOTROPIC: ("ff", "QQxx", "QQyx", "phi"), M.NEMATIC: ("ff", "QQxx", "QQyx")}


def whole(model, params, LX, LY, prec, st, steps):
    lat = M.Lattice(model, params, LX, LY, 0, prec)
    lat.upload_state(st)
    lat.step(steps)
    out = {k: lat.get(k) for k in FIELDS[model]}
    sums = lat.checks()
    lat.close()
    return out, sums


@pytest.mark.parametrize("model,params,LX,LY,prec,world", [
    (M.LYOTROPIC, LYO_ALL, 64, 128, M.FP32, 4),    # fused warp-strip kernel
    (M.LYOTROPIC, LYO_ALL, 50, 36, M.FP64, 3),     # FP64 sub-step kernels, uneven slabs
    (M.NEMATIC, NEM_ALL, 40, 64, M.FP32, 2),       # fused, nematic
    (M.LYOTROPIC, LYO_ALL, 36, 30, M.FP32, 4),     # FP32 unfused (LY % 4 != 0)
])
def test_emulated_ranks_equal_the_whole_lattice(model, params, LX, LY, prec, world):
    steps = 7
    st = O.synthetic_state(model, LX, LY, seed=31, flow=0.02)
    want, wsums = whole(model, params, LX, LY, prec, st, steps)
    slabs = [S.LatticeSlab(model, params, LX, LY, prec, x0, n)
             for x0, n in S.partition(LX, world)]
    for s in slabs:
        s.upload_global(st)
    if prec == M.FP32 and LY % 4 == 0:
        assert all(s.lat.uses_fused for s in slabs)
    ex = S.LocalExchange(slabs)
    ex.step(steps)
    for k in FIELDS[model]:
        assert bits_equal(ex.gather(k), want[k]), k
    f, p, bad = ex.checks()
    assert f == pytest.approx(wsums[0], rel=1e-12)
    assert p == pytest.approx(wsums[1], rel=1e-12, abs=1e-12)
    assert bad is False
    for s in slabs:
        s.close()


@pytest.mark.parametrize("prec", [M.FP64, M.FP32])
def test_single_rank_distributed_exchange(prec):
    LX, LY, steps = 48, 64, 5
    st = O.synthetic_state(M.LYOTROPIC, LX, LY, seed=8, flow=0.01)
    want, wsums = whole(M.LYOTROPIC, LYO_ALL, LX, LY, prec, st, steps)
    sl = S.LatticeSlab(M.LYOTROPIC, LYO_ALL, LX, LY, prec, 0, LX)
    sl.upload_global(st)
    run = S.SlabRun(sl, S.DistExchange())
    run.step(steps)
    for k in FIELDS[M.LYOTROPIC]:
        assert bits_equal(run.gather(k), want[k]), k
    f, p, bad = run.checks()
    assert f == pytest.approx(wsums[0], rel=1e-12)
    assert p == pytest.approx(wsums[1], rel=1e-12)
    sl.close()


def test_row_transfers_round_trip_and_refuse_bad_ranges():
    LX, LY = 24, 64
    st = O.synthetic_state(M.LYOTROPIC, LX, LY, seed=2)
    for prec in (M.FP32, M.FP64):
        lat = M.Lattice(M.LYOTROPIC, LYO_ALL, LX, LY, 0, prec)
        lat.upload_state(st)
        npl, eb = lat.rows_layout()
        assert npl == 12 and eb == (4 if prec == M.FP32 else 8)
        dt = torch.float32 if eb == 4 else torch.float64
        buf = torch.empty(npl * 5 * LY, dtype=dt, device="cuda")
        lat.get_rows(3, 5, buf.data_ptr())
        lat.synchronize()
        # the packed rows are the planes' rows 3..7
        q = buf.cpu().numpy().reshape(npl, 5, LY)
        assert np.array_equal(q[9].astype(np.float64),
                              lat.get("QQxx").reshape(LX, LY)[3:8])
        before = {k: lat.get(k) for k in ("ff", "QQxx", "phi")}
        lat.put_rows(10, 5, buf.data_ptr())
        after = {k: lat.get(k) for k in ("ff", "QQxx", "phi")}
        for k in after:
            a = after[k].reshape(LX, LY, -1)
            b = before[k].reshape(LX, LY, -1)
            assert bits_equal(a[10:15], b[3:8]), k
            assert bits_equal(a[:10], b[:10]) and bits_equal(a[15:], b[15:]), k
        f_all = lat.checks()[0]
        f_a = lat.checks_rows(0, 10)[0]
        f_b = lat.checks_rows(10, LX - 10)[0]
        assert f_a + f_b == pytest.approx(f_all, rel=1e-12)
        for x0, n in ((LX, 1), (0, 0), (20, 5)):
            with pytest.raises(M.MassLBError):
                lat.get_rows(x0, n, buf.data_ptr())
            with pytest.raises(M.MassLBError):
                lat.checks_rows(x0, n)
        lat.close()
    wall = M.Lattice(M.LYOTROPIC, LYO_ALL, LX, LY, 1, M.FP64)
    with pytest.raises(M.MassLBError):
        wall.get_rows(0, 4, buf.data_ptr())
    wall.close()


def test_step_rows_write_their_range_only():
    """mass_lb_set_step_rows: one step writes rows [x0, x0 + n) exactly as a
    whole-lattice step does, and leaves the other rows as they were two steps
    before (here: the uploaded state, since the ping-pong buffer holds it)."""
    LX, LY = 40, 128
    st = O.synthetic_state(M.LYOTROPIC, LX, LY, seed=8, flow=0.02)
    a = M.Lattice(M.LYOTROPIC, LYO_ALL, LX, LY, 0, M.FP32)
    b = M.Lattice(M.LYOTROPIC, LYO_ALL, LX, LY, 0, M.FP32)
    for x in (a, b):
        x.upload_state(st)
        x.step(1)       # both buffers now hold the first step
    a.set_step_rows(5, 23)
    a.step(1)
    b.step(1)
    for k in FIELDS[M.LYOTROPIC]:
        x = a.get(k).reshape(LX, LY, -1)
        y = b.get(k).reshape(LX, LY, -1)
        assert bits_equal(x[5:28], y[5:28]), k
    c0 = M.Lattice(M.LYOTROPIC, LYO_ALL, LX, LY, 0, M.FP32)
    c0.upload_state(st)
    for k in FIELDS[M.LYOTROPIC]:
        x = a.get(k).reshape(LX, LY, -1)
        s0 = c0.get(k).reshape(LX, LY, -1)
        assert bits_equal(x[:5], s0[:5]) and bits_equal(x[28:], s0[28:]), k
    a.set_step_rows(0, 0)
    a.step(1)
    # walls and npc > 1 refuse a row range
    w = M.Lattice(M.LYOTROPIC, LYO_ALL, 40, 128, 1, M.FP32)
    with pytest.raises(M.MassLBError):
        w.set_step_rows(4, 20)
    c = M.Lattice(M.LYOTROPIC, dict(LYO_ALL, npc=2), 40, 128, 0, M.FP32)
    with pytest.raises(M.MassLBError):
        c.set_step_rows(4, 20)
    with pytest.raises(M.MassLBError):
        a.set_step_rows(30, 20)
