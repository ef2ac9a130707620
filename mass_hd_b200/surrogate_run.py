"""Surrogate workloads: kernel timing, training, hybrid rollout.

    python -m mass_hd_b200.surrogate_run bench [--batch 32] [--size 256]
    python -m mass_hd_b200.surrogate_run train [--epochs 30] [--out weights.npz]
    python -m mass_hd_b200.surrogate_run hybrid --weights weights.npz [--steps 20000]

bench: CUDA-event time of each convolution kind at the training shape
(batch x size^2 pixels, 64 channels) and of one whole training step,
with the tensor-core rate against the measured bf16 peak.
train: simulator-generated dataset (40 trajectories of 256^2, zeta ~
U[0.005, 0.03], 50 (t, t+50) pairs each with t every 400 steps over
[2000, 22000), so 2000 pairs), AdamW with cosine learning rate, evaluation
on 4 held-out trajectories against persistence (prediction = input).
hybrid: plain LB against the hybrid loop on held-out trajectories
(`surrogate.hybrid`), simulated steps per second of each and the window
means of defect density and enstrophy density of both.
Each prints one JSON object.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np
import torch

from . import lb
from . import surrogate as G


def measured_peak_tflops():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                        "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def _time(fn, iters=20, warmup=3):
    for _ in range(warmup):
        fn()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(iters):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / iters


def mma_thread_cycles(net, L) -> dict:
    """Median over CTAs of the forward kernel's MMA-thread cycle counters
    (mass_sg_conv3x3_profile), for the GELU-epilogue convolution."""
    cyc = torch.zeros(4 * 1024, dtype=torch.int64, device="cuda")
    ncta = ctypes.c_int(0)
    G._call("mass_sg_conv3x3_profile", G._p(net.h[0]), G._p(L.wt), 64, G.FWD_GELU, net.B, net.H,
            net.W, G._p(L.b), None, None, G._p(net.u[0]), G._p(net.t[0]), None, None,
            G._p(net.err), G._p(cyc), ctypes.addressof(ncta), G._stream())
    torch.cuda.synchronize()
    c = cyc[:4 * ncta.value].view(-1, 4).cpu().numpy()
    med = np.median(c, axis=0)
    return {"ctas": ncta.value, "cycles_total": int(med[0]), "cycles_to_last_issue": int(med[1]),
            "waiting_for_slabs": int(med[2]), "waiting_for_accumulators": int(med[3])}


def bench(batch=32, size=256) -> dict:
    P = G.Params(seed=0)
    net = G.Net(P, batch, size, size, train=True)
    gen = torch.Generator(device="cuda").manual_seed(0)
    for t in [net.x_in] + net.h + net.u + net.t + [net.dout] + net.dh + [net.dt]:
        t.copy_(torch.randn(t.shape, generator=gen, device="cuda").to(torch.bfloat16))
    net.target.normal_(generator=gen)
    L = P.by_name["b0c1"]
    pix = batch * size * size
    flop = 2.0 * pix * 64 * 576
    out = {"batch": batch, "size": size, "pixels": pix, "gflop_per_conv": flop / 1e9}
    peak, kind = measured_peak_tflops()
    out["peak_tflops"], out["peak_kind"] = peak, kind
    cases = {
        "fwd_gelu": lambda: net._conv(net.h[0], L, G.FWD_GELU, out=net.u[0], out2=net.t[0]),
        "fwd_resid": lambda: net._conv(net.u[0], L, G.FWD_RESID, out=net.h[1], resid=net.h[0]),
        "dgrad_gelu": lambda: net._conv(net.dh[0], L, G.BWD_GELU, out=net.dt, aux=net.t[0],
                                        weights=L.wd),
        "wgrad": lambda: G._call("mass_sg_conv3x3_wgrad", G._p(net.h[0]), G._p(net.dt), G._p(L.dW),
                                 batch, size, size, G._p(net.err), G._stream()),
    }
    for k, fn in cases.items():
        ms = _time(fn)
        out[k] = {"ms": ms, "tflops": flop / ms / 1e9, "frac_of_peak": flop / ms / 1e9 / peak}
    out["fwd_gelu"]["mma_thread"] = mma_thread_cycles(net, L)

    def step():
        net.forward()
        net.backward()
        net.optimizer_step(1e-4)
    ms = _time(step, iters=10)
    nconv = 14 + 13 + 14
    out["train_step"] = {"ms": ms, "convs": nconv,
                         "tflops_effective": nconv * flop / ms / 1e9}
    ms = _time(net.forward, iters=10)
    out["forward"] = {"ms": ms, "images_per_s": batch / ms * 1e3}
    net.check_error_flag()
    return out


def train_cmd(epochs, out_path, seed=0, ntraj=40, heldout=4) -> dict:
    t0 = time.time()
    npairs = 50
    fields, zetas = G.generate_dataset(ntraj=ntraj + heldout, pairs=npairs, seed=seed)
    t_data = time.time() - t0
    n_train = ntraj * 2 * npairs
    mean, scale = G.normalise(fields[:n_train])
    fields[n_train:].sub_(torch.tensor(mean, device="cuda")).div_(torch.tensor(scale, device="cuda"))
    pairs = G.pair_indices(ntraj, npairs)
    test_pairs = G.pair_indices(heldout, npairs) + n_train
    P = G.Params(seed=seed)
    P.mean, P.scale = mean, scale
    t1 = time.time()
    losses = G.train(P, fields, pairs, epochs=epochs, batch=32, lr=1e-3, seed=seed,
                     log=lambda s: print(s, file=sys.stderr, flush=True))
    torch.cuda.synchronize()
    t_train = time.time() - t1
    ev = G.evaluate(P, fields, test_pairs)
    res = {"dataset_s": t_data, "train_s": t_train, "epochs": epochs, "pairs": int(len(pairs)),
           "params": P.count(), "losses": losses, "heldout": ev,
           "mean": mean.tolist(), "scale": scale.tolist()}
    if out_path:
        sd = P.state_dict()
        np.savez(out_path, mean=mean, scale=scale, **sd)
        res["weights"] = out_path
    return res


def load_params(path) -> G.Params:
    d = np.load(path)
    P = G.Params()
    P.load({k: d[k] for k in d.files if k.endswith(".w") or k.endswith(".b")})
    P.mean, P.scale = d["mean"].astype(np.float32), d["scale"].astype(np.float32)
    return P


def hybrid_cmd(weights, steps, M, threshold, nruns=8, seed=123, stats_every=1000) -> dict:
    P = load_params(weights)
    rng = np.random.default_rng(seed)
    zetas = rng.uniform(0.005, 0.03, nruns)
    states = [G.initial_state(256, rng) for _ in range(nruns)]

    def make():
        ens = lb.Ensemble(lb.LYOTROPIC, [G.training_params(z) for z in zetas], [(256, 256)] * nruns)
        for run, st in zip(ens.runs, states):
            run.upload_state(st)
        ens.step(2000)             # same spin-up as the training data
        return ens

    plain = make()
    torch.cuda.synchronize()
    samples_p = []
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        n = min(stats_every, steps - done)
        plain.step(n)
        done += n
        samples_p.append([r.statistics() for r in plain.runs])
    t_plain = time.perf_counter() - t0
    hyb = make()
    res_h = G.hybrid(P, hyb, steps, jump=50, M=M, threshold=threshold, stats_every=stats_every)

    def means(samples, window_from):
        sel = samples[max(window_from // stats_every - 1, 0):]
        N = 256 * 256
        dd = np.mean([[(x["defects_plus"] + x["defects_minus"]) / N for x in s] for s in sel])
        en = np.mean([[x["enstrophy_density"] for x in s] for s in sel])
        return {"defect_density": float(dd), "enstrophy_density": float(en)}

    win = steps // 2
    mp, mh = means(samples_p, win), means(res_h["samples"], win)
    errs = res_h["check_errors"]
    res = {"runs": nruns, "steps": steps, "M": M, "threshold": threshold,
           "plain_s": t_plain, "hybrid_s": res_h["wall_s"],
           "plain_steps_per_s": steps / t_plain, "hybrid_steps_per_s": steps / res_h["wall_s"],
           "speedup": t_plain / res_h["wall_s"],
           "surrogate_jumps": res_h["surrogate_jumps"],
           "plain_jumps_rejected": res_h["plain_jumps_rejected"], "checks": res_h["checks"],
           "nonfinite_rollouts": res_h["nonfinite_rollouts"],
           "check_error_median": float(np.median(errs)) if errs else None,
           "check_errors": [round(e, 4) for e in errs],
           "window_from": win, "plain_means": mp, "hybrid_means": mh,
           "rel_diff": {k: abs(mh[k] - mp[k]) / abs(mp[k]) if mp[k] else None for k in mp}}
    plain.close()
    hyb.close()
    return res


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    b = sub.add_parser("bench")
    b.add_argument("--batch", type=int, default=32)
    b.add_argument("--size", type=int, default=256)
    t = sub.add_parser("train")
    t.add_argument("--epochs", type=int, default=30)
    t.add_argument("--out", default=None)
    t.add_argument("--seed", type=int, default=0)
    h = sub.add_parser("hybrid")
    h.add_argument("--weights", required=True)
    h.add_argument("--steps", type=int, default=20000)
    h.add_argument("--M", type=int, default=10)
    h.add_argument("--threshold", type=float, default=0.5)
    h.add_argument("--runs", type=int, default=8)
    a = ap.parse_args(argv)
    if a.cmd == "bench":
        res = bench(a.batch, a.size)
    elif a.cmd == "train":
        res = train_cmd(a.epochs, a.out, a.seed)
    else:
        res = hybrid_cmd(a.weights, a.steps, a.M, a.threshold, a.runs)
    print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
