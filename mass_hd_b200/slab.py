"""One periodic lattice split into x-slabs, one per rank (GPU).

The reference steps one lattice in one process (its only mention of
distribution is the comment "Parallelization (MPI)" at src/models.hpp:15).
Here an LX x LY periodic lattice is cut along x, the slow index of the
reference's site order k = y + LY*x, so that each rank's rows are
contiguous in every plane:

* rank r of W owns rows [x0_r, x0_r + n_r) (`partition`), and holds them
  with HALO = 4 halo rows on each side as an ordinary periodic lattice of
  (n_r + 8) x LY sites: local row i is global row x0_r - 4 + i (mod LX);
* before every step the halo rows are refreshed from the neighbouring
  slabs (`DistExchange.exchange`): the first 4 owned rows go to the left
  neighbour's upper halo, the last 4 to the right neighbour's lower halo,
  each as one packed [plane][row][y] buffer (mass_lb_get_rows /
  mass_lb_put_rows on the device);
* one Step() reaches 4 rows along x - predictor UpdateQuantities (+-1),
  predictor UpdateFields with Move (+-1 each), corrector UpdateQuantities
  and UpdateFields (+-1 each) - so after the step the owned rows hold
  exactly what the whole lattice's step gives them, bit for bit, in FP64 and
  in FP32. The halo rows' own updates are wrong (their neighbourhood wraps
  inside the slab) and are overwritten by the next exchange;
* the conservation sums run over the owned rows (mass_lb_checks_rows) and
  are summed over ranks in FP64;
* a fused slab steps its owned rows only (mass_lb_set_step_rows); the
  halos' new values would be overwritten by the next exchange anyway.
  Slabs take npc = 1 (a step with npc correctors reaches 2 + 2*npc rows).

Transports: `DistExchange` sends the halo buffers with torch.distributed
point-to-point operations (NCCL between GPUs, into each GPU's own receive
buffer; gloo between CPU processes), one batch per step on the lattice's
stream. `LocalExchange` runs several slabs in one process (one GPU), the
ranks emulated as device-to-device copies. Neither uses peer loads or any
multicast.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

HALO = 4   # rows one Step() reaches along x


def partition(LX: int, world: int) -> List[Tuple[int, int]]:
    """(first row, rows) owned by each of `world` ranks: contiguous blocks,
    sizes differing by at most one. Every block must hold at least HALO
    rows, so that a halo comes from the immediate neighbour alone."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    base, extra = divmod(LX, world)
    out, x = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((x, n))
        x += n
    if world > 1 and min(n for _, n in out) < HALO:
        raise ValueError(f"{LX} rows over {world} ranks leaves a slab below {HALO} rows")
    return out


def check_npc(params: dict):
    """A step with npc correctors reaches 2 + 2*npc rows; the HALO rows
    cover npc = 1."""
    if int(params.get("npc", 1)) != 1:
        raise ValueError("x-slabs hold 4 halo rows, one step's reach with npc = 1")


def slab_rows(LX: int, x0: int, n: int) -> np.ndarray:
    """Global rows of a slab's local rows 0 .. n + 2*HALO - 1."""
    return (np.arange(-HALO, n + HALO) + x0) % LX


def local_state(state: dict, LX: int, LY: int, x0: int, n: int) -> dict:
    """The slab's (n + 2*HALO) x LY share of a global state in the
    reference's layout (ff as (LX*LY, 9), scalars as LX*LY)."""
    rows = slab_rows(LX, x0, n)
    out = {}
    for k, v in state.items():
        a = np.asarray(v)
        if a.ndim == 2:
            out[k] = a.reshape(LX, LY, a.shape[1])[rows].reshape(-1, a.shape[1])
        else:
            out[k] = a.reshape(LX, LY)[rows].reshape(-1)
    return out


def owned_part(arr: np.ndarray, n: int, LY: int) -> np.ndarray:
    """The owned rows of a slab-local field array."""
    a = np.asarray(arr)
    if a.ndim == 2:
        return a.reshape(-1, LY, a.shape[1])[HALO:HALO + n].reshape(-1, a.shape[1])
    return a.reshape(-1, LY)[HALO:HALO + n].reshape(-1)


class HaloBuffers:
    """Packed halo rows of one slab: send_lo (first owned rows, for the left
    neighbour), send_hi (last owned rows, for the right neighbour), recv_lo
    (the left neighbour's last rows, into the lower halo) and recv_hi (the
    right neighbour's first rows, into the upper halo)."""

    def __init__(self, nplanes: int, LY: int, dtype, device):
        import torch
        n = nplanes * HALO * LY
        self.send_lo = torch.empty(n, dtype=dtype, device=device)
        self.send_hi = torch.empty(n, dtype=dtype, device=device)
        self.recv_lo = torch.empty(n, dtype=dtype, device=device)
        self.recv_hi = torch.empty(n, dtype=dtype, device=device)
        self.bytes_per_exchange = 2 * n * self.send_lo.element_size()


class LatticeSlab:
    """A slab held by a Lattice of this library on the current device."""

    def __init__(self, model: int, params: dict, LX: int, LY: int, precision: int,
                 x0: int, n: int):
        import torch

        from mass_hd_b200 import lb
        check_npc(params)
        self.LX, self.LY, self.x0, self.n = LX, LY, x0, n
        self.lat = lb.Lattice(model, params, n + 2 * HALO, LY, 0, precision)
        if self.lat.uses_fused:
            # the halo rows' new values would be overwritten by the next
            # exchange: step the owned rows only (no partial chunk of the
            # 8 extra rows)
            self.lat.set_step_rows(HALO, n)
        self.nplanes, eb = self.lat.rows_layout()
        self.dtype = torch.float32 if eb == 4 else torch.float64
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.bufs = HaloBuffers(self.nplanes, LY, self.dtype, self.device)
        self._ext = torch.cuda.ExternalStream(self.lat.stream)

    def stream_context(self):
        import torch
        return torch.cuda.stream(self._ext)

    def upload_global(self, state: dict):
        self.lat.upload_state(local_state(state, self.LX, self.LY, self.x0, self.n))

    def get_rows(self, x0: int, nrows: int, out):
        self.lat.get_rows(x0, nrows, out.data_ptr())

    def put_rows(self, x0: int, nrows: int, src):
        self.lat.put_rows(x0, nrows, src.data_ptr())

    def step(self, k: int = 1):
        self.lat.step(k)

    def synchronize(self):
        self.lat.synchronize()

    def owned_sums(self):
        return self.lat.checks_rows(HALO, self.n)

    def owned(self, name: str) -> np.ndarray:
        return owned_part(self.lat.get(name), self.n, self.LY)

    def close(self):
        self.lat.close()


def pack_halos(slab):
    b = slab.bufs
    slab.get_rows(HALO, HALO, b.send_lo)       # first owned rows
    slab.get_rows(slab.n, HALO, b.send_hi)     # last owned rows


def unpack_halos(slab):
    b = slab.bufs
    slab.put_rows(0, HALO, b.recv_lo)
    slab.put_rows(slab.n + HALO, HALO, b.recv_hi)


class DistExchange:
    """Halo exchange of this rank's slab with its two neighbours over a
    torch.distributed process group (ranks ordered along x, periodic)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.rank = dist.get_rank(group)
            self.world = dist.get_world_size(group)
        else:   # a single process: the slab is the whole lattice
            self.rank, self.world = 0, 1

    def exchange(self, slab):
        import torch.distributed as dist
        b = slab.bufs
        pack_halos(slab)
        if self.world == 1:
            # the lattice's own periodic images
            b.recv_lo.copy_(b.send_hi)
            b.recv_hi.copy_(b.send_lo)
        else:
            left = (self.rank - 1) % self.world
            right = (self.rank + 1) % self.world
            g = lambda r: r if self.group is None else dist.get_global_rank(self.group, r)
            # tag 0: rows travelling left, tag 1: rows travelling right. The
            # same order on every rank also pairs them where tags are ignored
            # (NCCL matches each peer's operations in order).
            ops = [dist.P2POp(dist.isend, b.send_lo, g(left), self.group, 0),
                   dist.P2POp(dist.isend, b.send_hi, g(right), self.group, 1),
                   dist.P2POp(dist.irecv, b.recv_hi, g(right), self.group, 0),
                   dist.P2POp(dist.irecv, b.recv_lo, g(left), self.group, 1)]
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        unpack_halos(slab)

    def sum(self, values, device):
        import torch
        import torch.distributed as dist
        t = torch.tensor(list(values), dtype=torch.float64, device=device)
        if self.world > 1:
            dist.all_reduce(t, group=self.group)
        return [float(v) for v in t.tolist()]


class SlabRun:
    """This rank's share of one lattice, stepped with a halo exchange before
    every step. `slab` holds the rows (LatticeSlab on a GPU), `exchange`
    moves the halos (DistExchange)."""

    def __init__(self, slab, exchange: DistExchange):
        self.slab, self.ex = slab, exchange

    def step(self, k: int = 1):
        for _ in range(k):
            with self._ctx():
                self.ex.exchange(self.slab)
            self.slab.step(1)

    def _ctx(self):
        import contextlib
        ctx = getattr(self.slab, "stream_context", None)
        return ctx() if ctx else contextlib.nullcontext()

    def checks(self):
        """(population sum, phi sum, non-finite flag) over the whole lattice:
        each rank's owned rows, summed over ranks."""
        f, p, bad = self.slab.owned_sums()
        f, p, bad = self.ex.sum((f, p, float(bad)), self.slab.device)
        return f, p, bad != 0.0

    def gather(self, name: str):
        """The global field on rank 0 (None elsewhere), in the reference's
        layout."""
        import torch.distributed as dist
        part = self.slab.owned(name)
        if self.ex.world == 1:
            return part
        parts = [None] * self.ex.world if self.ex.rank == 0 else None
        dist.gather_object(part, parts, dst=0, group=self.ex.group)
        return np.concatenate(parts) if self.ex.rank == 0 else None


class LocalExchange:
    """Several slabs of one lattice in one process on one device (the ranks
    emulated): halos move by device-to-device copies between the slabs'
    buffers, after every slab's packing has finished."""

    def __init__(self, slabs: list):
        self.slabs = slabs

    def exchange_all(self):
        import torch
        W = len(self.slabs)
        for s in self.slabs:
            pack_halos(s)
        for s in self.slabs:
            s.synchronize()
        for r, s in enumerate(self.slabs):
            s.bufs.recv_lo.copy_(self.slabs[(r - 1) % W].bufs.send_hi)
            s.bufs.recv_hi.copy_(self.slabs[(r + 1) % W].bufs.send_lo)
        torch.cuda.synchronize()
        for s in self.slabs:
            unpack_halos(s)

    def step(self, k: int = 1):
        for _ in range(k):
            self.exchange_all()
            for s in self.slabs:
                s.step(1)

    def checks(self):
        tot = [0.0, 0.0, 0.0]
        for s in self.slabs:
            f, p, bad = s.owned_sums()
            tot[0] += f
            tot[1] += p
            tot[2] += float(bad)
        return tot[0], tot[1], tot[2] != 0.0

    def gather(self, name: str) -> np.ndarray:
        return np.concatenate([s.owned(name) for s in self.slabs])
