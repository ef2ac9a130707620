"""FP32 production mode against the FP64 mode, on the GPU.

    python -m mass_hd_b200.compare_precision [--model nematic] [--size 2048]
        [--field-steps 100] [--steps 5000] [--window 2000] [--every 100]

Both modes start from the same seeded state (random director with S=1, and
for lyotropic a tanh phi disk of radius L/4). Prints one JSON object:
  * per-field relative L2 difference after --field-steps steps
    (populations as deviations from t_v*rho);
  * for the statistics of mass_lb_statistics (defect density, <|u|^2>,
    enstrophy density, phi-interface length), the means over the steps
    window..steps sampled every --every steps in each mode, and their
    relative difference. Active turbulence is chaotic, so long runs are
    compared through these window means, not field by field.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from mass_hd_b200 import lb
from mass_hd_b200.run_case import PARAMS, REST, seeded_state

STATS = ("defect_density", "mean_u2", "enstrophy_density", "perimeter")


def rel_l2(a, b) -> float:
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a - b))


def field_errors(a: lb.Lattice, b: lb.Lattice, model: str, rho: float = 40.0) -> dict:
    out = {}
    names = ("ff", "QQxx", "QQyx") + (("phi",) if model == "lyotropic" else ())
    for n in names:
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = x - REST * rho, y - REST * rho
        out[n] = rel_l2(x, y)
    return out


def stat_sample(lat: lb.Lattice) -> dict:
    s = lat.statistics()
    N = lat.LX * lat.LY
    return {"defect_density": (s["defects_plus"] + s["defects_minus"]) / N,
            "mean_u2": s["mean_u2"], "enstrophy_density": s["enstrophy_density"],
            "perimeter": s["perimeter"]}


def compare(model: str, size: int, field_steps: int, steps: int, window: int, every: int,
            seed: int = 1) -> dict:
    mcode = lb.LYOTROPIC if model == "lyotropic" else lb.NEMATIC
    st = seeded_state(model, size, seed)
    a = lb.Lattice(mcode, PARAMS[model], size, size, 0, lb.FP32)
    b = lb.Lattice(mcode, PARAMS[model], size, size, 0, lb.FP64)
    a.upload_state(st)
    b.upload_state(st)
    t0 = time.time()
    a.step(field_steps)
    b.step(field_steps)
    out = {"model": model, "size": size, "field_steps": field_steps,
           "field_rel_l2": field_errors(a, b, model)}
    samples = {"fp32": [], "fp64": []}
    t = field_steps
    while t < steps:
        n = every - (t % every) if t % every else every
        n = min(n, steps - t)
        a.step(n)
        b.step(n)
        t += n
        if t >= window and t % every == 0:
            samples["fp32"].append(stat_sample(a))
            samples["fp64"].append(stat_sample(b))
    win = {}
    for k in STATS:
        m32 = float(np.mean([s[k] for s in samples["fp32"]])) if samples["fp32"] else float("nan")
        m64 = float(np.mean([s[k] for s in samples["fp64"]])) if samples["fp64"] else float("nan")
        win[k] = {"fp32": m32, "fp64": m64,
                  "rel_diff": abs(m32 - m64) / abs(m64) if m64 else abs(m32 - m64)}
    out["window"] = {"from": window, "to": steps, "every": every, "samples": len(samples["fp32"]),
                     "means": win}
    out["seconds"] = time.time() - t0
    a.close()
    b.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--model", default="nematic", choices=sorted(PARAMS))
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--field-steps", type=int, default=100)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--window", type=int, default=2000)
    ap.add_argument("--every", type=int, default=100)
    a = ap.parse_args(argv)
    print(json.dumps(compare(a.model, a.size, a.field_steps, a.steps, a.window, a.every)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
