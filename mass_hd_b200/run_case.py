"""Run a seeded lattice for a number of steps through the C ABI.

    python -m mass_hd_b200.run_case [--model lyotropic|nematic|go-or-grow]
        [--size L] [--steps N] [--precision fp32|fp64] [--tile THREADS,ROWS]

A small self-contained case for profilers and quick checks: uploads the
seeded synthetic state (random director with S=1; for lyotropic a tanh phi
disk of radius L/4; for go-or-grow the same disk with m = phi and a growth
rate on every 7th site with phi >= 0.5), runs N steps, prints the tile and
the conservation sums.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))

from mass_hd_b200 import lb  # noqa: E402

PARAMS = {
    "lyotropic": dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5, tauIso=1.5, rho=40.0,
                      friction=0.0, AA=0.1, CC=0.1, LL=0.05, KK=0.05, zeta=0.01,
                      zetaI=0.0, conc=1.0, npc=1),
    "nematic": dict(Gamma=0.3, xi=0.7, tau=1.5, rho=40.0, friction=0.0, CC=0.1,
                    LL=0.05, zeta=0.02, npc=1),
    # go-or-grow with the physics of the reference's cases/test/test.dat
    "go-or-grow": dict(GammaQ=0.3, GammaP=5e-2, xi=0.3, tauNem=1.0, tauIso=1.0, rho=40.0,
                       friction=0.0, AA=0.03, CC=0.1, LL=0.002, KK=0.06, zeta=0.0, zetaI=0.0,
                       conc=1.0, npc=1, B=0.1, Snem=1.0, alpha=0.001,
                       **{"phi-critical": 1.2}),
}
MODELS = {"lyotropic": lb.LYOTROPIC, "nematic": lb.NEMATIC, "go-or-grow": lb.GO_OR_GROW}
REST = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def seeded_state(model: str, L: int, seed: int = 1, rho: float = 40.0) -> dict:
    rng = np.random.default_rng(seed)
    theta = rng.uniform(0.0, np.pi, L * L)
    st = {"QQxx": np.cos(2 * theta), "QQyx": np.sin(2 * theta),
          "ff": np.tile(REST * rho, (L * L, 1))}
    if model != "nematic":
        x = np.arange(L)[:, None] - L / 2
        y = np.arange(L)[None, :] - L / 2
        r = np.sqrt(x * x + y * y).reshape(-1)
        st["phi"] = 0.5 * (1 - np.tanh((r - L / 4) / 2))
    if model == "go-or-grow":
        st["m"] = np.maximum(st["phi"], 0.0)
    return st


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--model", default="lyotropic", choices=sorted(PARAMS))
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--tile", default=None, help="THREADS,ROWS of the fused kernel")
    a = ap.parse_args(argv)
    mcode = MODELS[a.model]
    prec = lb.FP32 if a.precision == "fp32" else lb.FP64
    lat = lb.Lattice(mcode, PARAMS[a.model], a.size, a.size, 0, prec)
    if a.tile and lat.uses_fused:
        t, r = (int(v) for v in a.tile.split(","))
        lat.set_tile(t, r)
    st = seeded_state(a.model, a.size)
    lat.upload_state(st)
    if a.model == "go-or-grow":
        grow = (st["phi"] >= 0.5) & (np.arange(a.size * a.size) % 7 == 0)
        lat.set_phi_source(np.where(grow, PARAMS[a.model]["alpha"], 0.0))
    lat.step(a.steps)
    lat.synchronize()
    f, p, bad = lat.checks()
    tile = lat.tile() if lat.uses_fused else None
    print(f"{a.model} {a.size}^2 {a.precision}: {a.steps} steps, tile {tile}, "
          f"sum f {f:.6f}, sum phi {p:.6f}, nonfinite {bad}")
    lat.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
