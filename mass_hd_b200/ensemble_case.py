"""Batched parameter sweep: many lyotropic runs of uneven size advanced together.

    python -m mass_hd_b200.ensemble_case [--runs 96] [--steps 1000] [--seed 7]
    torchrun --nproc-per-node N -m mass_hd_b200.ensemble_case --sharded [...]

The sweep: each run's lattice is L x L with L drawn uniformly from
{128, 192, 256, 384, 512}; zeta log-uniform in [1e-3, 5e-2]; the nematic
elastic constant LL uniform in [0.02, 0.08]; xi from {0.3, 0.7, 1.0}; the
initial phi a tanh disk of radius L/4 or random phi with mean 0.5 and sd 0.05
(one or the other with equal odds); a random director with S = 1.

The script advances the same seeded runs twice, from the same states: once
through the ensemble (one persistent launch per step for all runs,
mass_lb_ensemble_step) and once run after run through the single-lattice
path (mass_lb_step, autotuned tile per run), checks that both give
bit-identical states, and prints one JSON object with both times and their
ratio. Timing is wall-clock around device-synchronised calls.

--sharded (one process per GPU): the runs are independent, so they are
split over the ranks with no communication on the data path
(`partition_runs`: largest lattice first onto the rank with the fewest
sites so far), each rank steps its share as one ensemble, and the time is
the slowest rank's (an all-reduce of one number). Rank 0 prints the sites,
the per-rank loads and the whole job's site-updates per second.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from mass_hd_b200 import lb
from mass_hd_b200.run_case import PARAMS, REST

SIZES = (128, 192, 256, 384, 512)
XI = (0.3, 0.7, 1.0)


def sweep(nruns: int = 96, seed: int = 7, sizes=SIZES):
    """[(params, (L, L), state)] for the sweep described in the module docstring."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nruns):
        L = int(rng.choice(sizes))
        p = dict(PARAMS["lyotropic"])
        p["zeta"] = float(np.exp(rng.uniform(np.log(1e-3), np.log(5e-2))))
        p["LL"] = float(rng.uniform(0.02, 0.08))
        p["xi"] = float(rng.choice(XI))
        theta = rng.uniform(0.0, np.pi, L * L)
        st = {"QQxx": np.cos(2 * theta), "QQyx": np.sin(2 * theta),
              "ff": np.tile(REST * p["rho"], (L * L, 1))}
        if rng.uniform() < 0.5:
            x = np.arange(L)[:, None] - L / 2
            y = np.arange(L)[None, :] - L / 2
            r = np.sqrt(x * x + y * y).reshape(-1)
            st["phi"] = 0.5 * (1 - np.tanh((r - 0.25 * L) / 2))
        else:
            st["phi"] = rng.normal(0.5, 0.05, L * L)
        out.append((p, (L, L), st))
    return out


def partition_runs(sizes, world: int):
    """Run indices per rank: runs sorted by site count, largest first, each
    given to the rank with the fewest sites so far (ties to the lowest
    rank). Every run lands on exactly one rank; the loads differ by at most
    the largest run."""
    load = [0] * world
    share = [[] for _ in range(world)]
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i][0] * sizes[i][1], i))
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        share[r].append(i)
        load[r] += sizes[i][0] * sizes[i][1]
    return [sorted(x) for x in share], load


def run_sharded(nruns: int, steps: int, seed: int = 7) -> dict:
    """This rank's share of the sweep as one ensemble (see --sharded)."""
    import os

    import torch

    import bench
    rank, world, local = bench.dist_setup(int(os.environ.get("WORLD_SIZE", "1")))
    torch.cuda.set_device(local)
    cases = sweep(nruns, seed)
    share, load = partition_runs([c[1] for c in cases], world)
    mine = [cases[i] for i in share[rank]]
    t = 0.0
    if mine:
        ens, t = run_batched(mine, steps)
        ens.close()
    t_max = bench.max_over_ranks(t, world)
    out = {"runs": nruns, "steps": steps, "ranks": world, "rank_sites": load,
           "rank_runs": [len(x) for x in share], "slowest_rank_s": t_max,
           "site_updates_per_s": site_updates(cases, steps) / t_max if t_max > 0 else None}
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return out if rank == 0 else None


def site_updates(cases, steps: int) -> int:
    return steps * sum(s[0] * s[1] for _, s, _ in cases)


def run_batched(cases, steps: int, warmup: int = 2):
    ens = lb.Ensemble(lb.LYOTROPIC, [c[0] for c in cases], [c[1] for c in cases])
    for run, (_, _, st) in zip(ens.runs, cases):
        run.upload_state(st)
    ens.step(warmup)            # picks the chunk height, builds the graph
    t0 = time.perf_counter()
    ens.step(steps)
    dt = time.perf_counter() - t0
    return ens, dt


def run_sequential(cases, steps: int, warmup: int = 2):
    lats = []
    for p, (LX, LY), st in cases:
        lat = lb.Lattice(lb.LYOTROPIC, p, LX, LY, 0, lb.FP32)
        lat.upload_state(st)
        lat.step(warmup)        # autotunes the tile of this lattice
        lat.synchronize()
        lats.append(lat)
    t0 = time.perf_counter()
    for lat in lats:
        lat.step(steps)
        lat.synchronize()
    dt = time.perf_counter() - t0
    return lats, dt


def compare(nruns: int, steps: int, seed: int = 7) -> dict:
    cases = sweep(nruns, seed)
    ens, t_b = run_batched(cases, steps)
    lats, t_s = run_sequential(cases, steps)
    identical = all(np.array_equal(r.get(n), s.get(n))
                    for r, s in zip(ens.runs, lats) for n in ("ff", "QQxx", "QQyx", "phi"))
    n = site_updates(cases, steps + 2)
    out = {"runs": nruns, "steps": steps, "sites": site_updates(cases, 1),
           "batched_s": t_b, "sequential_s": t_s, "speedup": t_s / t_b,
           "batched_site_updates_per_s": site_updates(cases, steps) / t_b,
           "sequential_site_updates_per_s": site_updates(cases, steps) / t_s,
           "ensemble_rows": ens.rows, "bit_identical": bool(identical),
           "total_site_updates": n}
    ens.close()
    for lat in lats:
        lat.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=96)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--sharded", action="store_true",
                    help="split the runs over the ranks of a torchrun launch")
    a = ap.parse_args(argv)
    if a.sharded:
        r = run_sharded(a.runs, a.steps, a.seed)
        if r is not None:
            print(json.dumps(r))
        return 0
    print(json.dumps(compare(a.runs, a.steps, a.seed)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
