"""x-slab decomposition of one lattice over ranks, on the CPU (gloo).

mass_hd_b200/slab.py splits an LX x LY periodic lattice into x-slabs with 4
halo rows on each side and refreshes the halos before every step. Here each
rank steps its slab with the FP64 C restatement of Step() (the oracle, which
is pinned bit for bit to the reference's own build), the halos travel over
gloo with the same exchange code the GPU ranks use over NCCL, and the owned
rows gathered on rank 0 must equal the whole lattice stepped in one process,
bit for bit. Also: the partition, the conservation sums over ranks, and a
world of three ranks whose slabs are uneven.
"""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from mass_hd_b200 import slab as S
from oracle import oracle as O
from tests.helpers import LYO_ALL, NEM_ALL

PLANES = {O.LYOTROPIC: ("QQxx", "QQyx", "phi"), O.NEMATIC: ("QQxx", "QQyx")}


class OracleSlab:
    """A slab stepped by the FP64 oracle, packing rows like mass_lb_get_rows
    ([plane][row][y]: 9 populations, Qxx, Qyx, phi)."""

    def __init__(self, model, params, LX, LY, x0, n, state):
        import torch
        self.model, self.LY, self.n = model, LY, n
        self.o = O.PortOracle(model, params, n + 2 * S.HALO, LY, 0)
        for k, v in S.local_state(state, LX, LY, x0, n).items():
            self.o.set(k, v)
        self.nplanes = 9 + len(PLANES[model])
        self.device = torch.device("cpu")
        self.bufs = S.HaloBuffers(self.nplanes, LY, torch.float64, self.device)

    def _planes(self):
        ff = self.o.get("ff").reshape(-1, self.LY, 9)
        out = [ff[:, :, v] for v in range(9)]
        out += [self.o.get(k).reshape(-1, self.LY) for k in PLANES[self.model]]
        return out

    def get_rows(self, x0, nrows, out):
        import torch
        rows = np.stack([p[x0:x0 + nrows] for p in self._planes()])
        out.copy_(torch.from_numpy(rows.reshape(-1)))

    def put_rows(self, x0, nrows, src):
        a = src.numpy().reshape(self.nplanes, nrows, self.LY)
        ff = self.o.get("ff").reshape(-1, self.LY, 9)
        for v in range(9):
            ff[x0:x0 + nrows, :, v] = a[v]
        self.o.set("ff", ff.reshape(-1, 9))
        for i, k in enumerate(PLANES[self.model]):
            f = self.o.get(k).reshape(-1, self.LY)
            f[x0:x0 + nrows] = a[9 + i]
            self.o.set(k, f.reshape(-1))

    def step(self, k=1):
        self.o.step(k)

    def owned(self, name):
        return S.owned_part(self.o.get(name), self.n, self.LY)

    def owned_sums(self):
        ff = self.owned("ff")
        phi = self.owned("phi").sum() if self.model == O.LYOTROPIC else 0.0
        return float(ff.sum()), float(phi), False


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _params(model):
    return LYO_ALL if model == O.LYOTROPIC else NEM_ALL


def _global_state(model, LX, LY):
    return O.synthetic_state(model, LX, LY, seed=23, flow=0.02)


def _rank_main(rank, world, port, model, LX, LY, steps, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        x0, n = S.partition(LX, world)[rank]
        sl = OracleSlab(model, _params(model), LX, LY, x0, n, _global_state(model, LX, LY))
        run = S.SlabRun(sl, S.DistExchange())
        run.step(steps)
        sums = run.checks()
        fields = {k: run.gather(k) for k in ("ff",) + PLANES[model]}
        q.put((rank, sums, fields if rank == 0 else None, None))
    except Exception as e:   # report instead of hanging the other rank
        q.put((rank, None, None, repr(e)))
    finally:
        dist.destroy_process_group()


def _run_world(world, model, LX, LY, steps):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, model, LX, LY, steps, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, _, _, err in out:
        assert err is None, (r, err)
    return sorted(out, key=lambda o: o[0])


@pytest.mark.parametrize("world,model,LX,LY", [(2, O.LYOTROPIC, 20, 12),
                                               (3, O.LYOTROPIC, 14, 10),
                                               (2, O.NEMATIC, 16, 14)])
def test_slabs_step_like_the_whole_lattice(world, model, LX, LY):
    steps = 5
    out = _run_world(world, model, LX, LY, steps)
    ref = O.PortOracle(model, _params(model), LX, LY, 0)
    for k, v in _global_state(model, LX, LY).items():
        ref.set(k, v)
    ref.step(steps)
    fields = out[0][2]
    for k in ("ff",) + PLANES[model]:
        assert np.array_equal(fields[k], ref.get(k)), k
    # the same global sums on every rank, equal to the whole lattice's
    f_all = float(ref.get("ff").sum())
    for _, sums, _, _ in out:
        assert sums == out[0][1]
        assert sums[0] == pytest.approx(f_all, rel=1e-13)
        if model == O.LYOTROPIC:
            assert sums[1] == pytest.approx(float(ref.get("phi").sum()), rel=1e-13)
        assert sums[2] is False


def test_partition_covers_every_row_once():
    for LX in (8, 9, 31, 4096, 8192):
        for W in (1, 2, 3, 8):
            if LX // W < S.HALO and W > 1:
                with pytest.raises(ValueError):
                    S.partition(LX, W)
                continue
            parts = S.partition(LX, W)
            assert parts[0][0] == 0
            assert sum(n for _, n in parts) == LX
            for (a, n), (b, _) in zip(parts, parts[1:]):
                assert a + n == b
            assert max(n for _, n in parts) - min(n for _, n in parts) <= 1


def test_slab_rows_wrap_periodically():
    assert list(S.slab_rows(10, 0, 3)) == [6, 7, 8, 9, 0, 1, 2, 3, 4, 5, 6]
    st = {"phi": np.arange(12.0), "ff": np.arange(24.0).reshape(12, 2)}
    loc = S.local_state(st, 6, 2, 4, 2)
    # rows 0, 1, ..., of the slab: global rows 0, 1, 2, 3, 4, 5, 0, 1, 2, 3
    assert list(loc["phi"][:4]) == [0.0, 1.0, 2.0, 3.0]
    assert S.owned_part(loc["phi"], 2, 2).tolist() == [8.0, 9.0, 10.0, 11.0]
    assert S.owned_part(loc["ff"], 2, 2).shape == (4, 2)


def test_ensemble_runs_split_over_ranks_once_and_balanced():
    from mass_hd_b200 import ensemble_case as E
    cases = E.sweep(96, seed=7)
    sizes = [c[1] for c in cases]
    for world in (1, 2, 3, 8):
        share, load = E.partition_runs(sizes, world)
        flat = sorted(i for s in share for i in s)
        assert flat == list(range(96))
        assert load == [sum(sizes[i][0] * sizes[i][1] for i in s) for s in share]
        assert max(load) - min(load) <= 512 * 512
    # more ranks than runs: some ranks get nothing, none gets a run twice
    share, load = E.partition_runs([(128, 128), (256, 256)], 4)
    assert sorted(i for s in share for i in s) == [0, 1] and load.count(0) == 2


def test_slabs_take_one_corrector():
    S.check_npc({"npc": 1})
    S.check_npc({})
    with pytest.raises(ValueError):
        S.check_npc({"npc": 2})
