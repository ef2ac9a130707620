"""One large lattice, plain method against the surrogate hybrid.

    python -m mass_hd_b200.c5_run [--size 8192] [--steps 50000] [--every 1000]
        [--M 10] [--threshold 1.0] [--epochs 30] [--weights PATH]

The workload: a lyotropic 8192^2 periodic lattice (zeta 0.02, LL 0.05,
xi 0.7, the other terms of the 256^2 configuration), random director with
S = 1 and phi ~ N(0.5, 0.05) i.i.d., 50k steps, in FP32.

1. The surrogate is trained on 256^2 trajectories started the same way
   (random phi), zeta ~ U[0.015, 0.025] around the run's 0.02 (or loaded
   from --weights, as surrogate_run writes them).
2. Plain: the lattice is stepped to `steps`, with the flow, defect and
   interface statistics (mass_lb_statistics) every `every` steps.
3. Hybrid: the same seeded start, `spinup` plain steps (the training data
   begin there), then surrogate.hybrid_tiled: the network applied tile by
   tile with circular halos (surrogate.TiledSurrogate), re-synchronised by
   one plain jump every M jumps.
4. Window means over the second half of the run of defect density,
   <|u|^2>, enstrophy density and phi-interface length, plain against
   hybrid, with both wall times, the jumps each method took and the cost of
   one surrogate prediction of the whole lattice against one plain jump.

Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np
import torch

from . import lb
from . import surrogate as G
from .long_run import initial_state
from .run_case import PARAMS

STATS = ("defect_density", "mean_u2", "enstrophy_density", "perimeter")


def c5_params(zeta=0.02, LL=0.05, xi=0.7) -> dict:
    return dict(PARAMS["lyotropic"], zeta=zeta, LL=LL, xi=xi)


def stat_row(s: dict, N: int) -> dict:
    return {"defect_density": (s["defects_plus"] + s["defects_minus"]) / N,
            "mean_u2": s["mean_u2"], "enstrophy_density": s["enstrophy_density"],
            "perimeter": s["perimeter"]}


def train_random_phi(epochs: int, seed: int = 0, ntraj: int = 40) -> G.Params:
    npairs = 50
    fields, _ = G.generate_dataset(ntraj=ntraj, pairs=npairs, seed=seed,
                                   zeta_range=(0.015, 0.025), phi="random")
    mean, scale = G.normalise(fields)
    P = G.Params(seed=seed)
    P.mean, P.scale = mean, scale
    G.train(P, fields, G.pair_indices(ntraj, npairs), epochs=epochs, batch=32, lr=1e-3,
            seed=seed)
    del fields
    torch.cuda.empty_cache()
    return P


def run(size, steps, every, M, threshold, epochs, weights, seed=1, spinup=2000) -> dict:
    t0 = time.time()
    if weights:
        from .surrogate_run import load_params
        P = load_params(weights)
    else:
        P = train_random_phi(epochs)
    t_train = time.time() - t0
    N = size * size
    st = initial_state(size, "random", seed)
    p = c5_params()

    # plain
    lat = lb.Lattice(lb.LYOTROPIC, p, size, size, 0, lb.FP32)
    lat.upload_state(st)
    lat.step(1)
    lat.synchronize()
    plain = []
    t1 = time.perf_counter()
    done = 1
    while done < steps:
        n = min(every - done % every, steps - done)
        lat.step(n)
        done += n
        plain.append((done, stat_row(lat.statistics(), N)))
    lat.synchronize()
    t_plain = time.perf_counter() - t1
    plain_ms_per_step = 1e3 * t_plain / (steps - 1)
    lat.close()

    # hybrid from the same start
    lat = lb.Lattice(lb.LYOTROPIC, p, size, size, 0, lb.FP32)
    lat.upload_state(st)
    lat.step(spinup)
    lat.synchronize()
    tiler = G.TiledSurrogate(P, size, size)
    # the cost of one surrogate prediction of the whole lattice
    G.fields_from_lattice(lat, tiler.cur, P.mean, P.scale)
    tiler.predict(tiler.cur, tiler.pred)
    torch.cuda.synchronize()
    tp = time.perf_counter()
    tiler.predict(tiler.cur, tiler.pred)
    torch.cuda.synchronize()
    predict_s = time.perf_counter() - tp
    span = (steps - spinup) // (50 * M) * 50 * M
    res = G.hybrid_tiled(P, lat, span, jump=50, M=M, threshold=threshold, stats_every=every,
                         tiler=tiler)
    hybrid = [(spinup + t, stat_row(s, N)) for t, s in res["samples"]]
    lat.close()

    win = steps // 2

    def means(series):
        sel = [s for t, s in series if t >= win]
        return {k: float(np.mean([s[k] for s in sel])) for k in STATS}, len(sel)

    mp, npl = means(plain)
    mh, nhy = means(hybrid)
    # plain time over the hybrid's span (spin-up excluded from both)
    plain_span_s = plain_ms_per_step * span / 1e3
    return {
        "size": size, "steps": steps, "spinup": spinup, "M": M, "threshold": threshold,
        "train_s": t_train,
        "plain_ms_per_step": plain_ms_per_step,
        "plain_site_updates_per_s": N / (plain_ms_per_step / 1e3),
        "surrogate_predict_ms": 1e3 * predict_s,
        "plain_jump_ms": 50 * plain_ms_per_step,
        "hybrid_span_steps": span, "hybrid_s": res["wall_s"], "plain_span_s": plain_span_s,
        "speedup": plain_span_s / res["wall_s"],
        "surrogate_jumps": res["surrogate_jumps"],
        "plain_jumps_rejected": res["plain_jumps_rejected"], "checks": res["checks"],
        "nonfinite_rollouts": res["nonfinite_rollouts"],
        "check_error_median": float(np.median(res["check_errors"])),
        "check_errors": [round(e, 4) for e in res["check_errors"]],
        "window_from": win, "samples": {"plain": npl, "hybrid": nhy},
        "plain_means": mp, "hybrid_means": mh,
        "rel_diff": {k: abs(mh[k] - mp[k]) / abs(mp[k]) if mp[k] else None for k in STATS},
        "plain_series": plain, "hybrid_series": hybrid,
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=8192)
    ap.add_argument("--steps", type=int, default=50000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--M", type=int, default=10)
    ap.add_argument("--threshold", type=float, default=1.0)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--weights", default=None)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.size, a.steps, a.every, a.M, a.threshold, a.epochs, a.weights)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
