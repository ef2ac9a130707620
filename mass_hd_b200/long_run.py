"""A long run with on-GPU statistics instead of frame files.

    python -m mass_hd_b200.long_run [--size 8192] [--steps 50000] [--every 1000]
        [--precision fp32] [--phi random] [--zeta 0.02] [--seed 1]

The state starts from a seeded random director (S = 1) and either random
phi ~ N(0.5, 0.05) (`--phi random`, the 8192^2 workload) or a tanh disk of
radius L/4 (`--phi disk`). Every `--every` steps the run takes the
runtime checks (population and phi totals, non-finite values) and the flow
and defect statistics (mass_lb_statistics) on the device; it prints one
JSON object with the throughput (CUDA events around the stepping only),
the time spent in checks and statistics, and the statistics time series.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np
import torch

from . import lb
from .run_case import PARAMS, REST


def initial_state(L: int, phi: str, seed: int, conc: float = 0.5, sd: float = 0.05) -> dict:
    rng = np.random.default_rng(seed)
    theta = rng.uniform(0.0, np.pi, L * L)
    st = {"QQxx": np.cos(2 * theta), "QQyx": np.sin(2 * theta),
          "ff": np.tile(REST * 40.0, (L * L, 1))}
    if phi == "random":
        st["phi"] = rng.normal(conc, sd, L * L)
    else:
        x = np.arange(L)[:, None] - L / 2
        y = np.arange(L)[None, :] - L / 2
        r = np.sqrt(x * x + y * y).reshape(-1)
        st["phi"] = 0.5 * (1 - np.tanh((r - L / 4) / 2))
    return st


def run(size, steps, every, precision, phi, zeta, seed, LL=0.05, xi=0.7) -> dict:
    p = dict(PARAMS["lyotropic"], zeta=zeta, LL=LL, xi=xi)
    prec = lb.FP32 if precision == "fp32" else lb.FP64
    lat = lb.Lattice(lb.LYOTROPIC, p, size, size, 0, prec)
    t0 = time.time()
    lat.upload_state(initial_state(size, phi, seed))
    t_upload = time.time() - t0
    lat.step(1)                      # autotunes the tile before timing
    lat.synchronize()
    stream = torch.cuda.ExternalStream(lat.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms = 0.0
    host_s = 0.0
    series = []
    done = 1
    N = size * size
    while done < steps:
        n = min(every - done % every, steps - done)   # up to the next multiple of `every`
        e0.record(stream)
        lat.step(n)
        e1.record(stream)
        e1.synchronize()
        step_ms += e0.elapsed_time(e1)
        done += n
        h0 = time.time()
        f, ptot = lat.runtime_checks()
        s = lat.statistics()
        host_s += time.time() - h0
        series.append({"step": done, "fsum": f, "phisum": ptot,
                       "defect_density": (s["defects_plus"] + s["defects_minus"]) / N,
                       "mean_u2": s["mean_u2"], "enstrophy_density": s["enstrophy_density"],
                       "perimeter": s["perimeter"], "phi_area": s["phi_area"]})
    timed_steps = done - 1
    out = {"size": size, "steps": done, "precision": precision, "phi": phi, "zeta": zeta,
           "tile": list(lat.tile()) if lat.uses_fused else None,
           "ms_per_step": step_ms / timed_steps,
           "site_updates_per_s": N * timed_steps / (step_ms / 1e3),
           "upload_s": t_upload, "checks_and_stats_s": host_s,
           "checks_and_stats_per_sample_ms": 1e3 * host_s / max(len(series), 1),
           "ftot": lat.initial_totals()[0], "series": series}
    lat.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--steps", type=int, default=50000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--phi", default="random", choices=["random", "disk"])
    ap.add_argument("--zeta", type=float, default=0.02)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.size, a.steps, a.every, a.precision, a.phi, a.zeta, a.seed)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
