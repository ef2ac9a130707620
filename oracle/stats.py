"""CPU restatement of the flow/defect statistics (test infrastructure only).

Restates, in numpy, the estimators of the reference's post-processing that
mass_lb_statistics computes on the device; pinned against values produced
by the reference's own code (tests/golden/gen_stats_golden.py):
  * velocity from the populations
    (plot/python/passive_q1_alpha_regime_analysis.py:137-145);
  * vorticity by periodic central differences (:148-151) and enstrophy
    density 0.5 <w^2> (:339-348);
  * perimeter_4 of phi > 0.5 with the lattice edge exposed (:206-216);
  * director from Q (POST/massPy/nematic/nematicPy.py:4-15), winding of the
    director around each site's 8-site ring with the nematic fold
    (POST/massPy/base_modules/defects.py:15-50), and +-1/2 defects as
    4-connected same-sign clusters of |charge| > 0.4 (defects.py:58-110).
"""
from __future__ import annotations

import numpy as np


def velocity(ff: np.ndarray, LX: int, LY: int, rest: float = 0.0):
    f = np.asarray(ff, dtype=float).reshape(-1, 9)
    rho = rest + f.sum(axis=1)
    jx = f[:, 1] - f[:, 2] + f[:, 5] - f[:, 6] - f[:, 7] + f[:, 8]
    jy = f[:, 3] - f[:, 4] + f[:, 5] - f[:, 6] + f[:, 7] - f[:, 8]
    with np.errstate(divide="ignore", invalid="ignore"):
        vx = np.where(rho == 0, 0.0, jx / rho)
        vy = np.where(rho == 0, 0.0, jy / rho)
    return vx.reshape(LX, LY), vy.reshape(LX, LY)


def vorticity(vx: np.ndarray, vy: np.ndarray) -> np.ndarray:
    dvdx = 0.5 * (np.roll(vy, -1, axis=0) - np.roll(vy, 1, axis=0))
    dudy = 0.5 * (np.roll(vx, -1, axis=1) - np.roll(vx, 1, axis=1))
    return dvdx - dudy


def perimeter_4(mask: np.ndarray) -> float:
    p = np.pad(mask.astype(bool), 1, constant_values=False)
    c = p[1:-1, 1:-1]
    return float(np.sum(c & ~p[2:, 1:-1]) + np.sum(c & ~p[:-2, 1:-1])
                 + np.sum(c & ~p[1:-1, 2:]) + np.sum(c & ~p[1:-1, :-2]))


def charge(Qxx: np.ndarray, Qyx: np.ndarray, LX: int, LY: int) -> np.ndarray:
    Qxx = np.asarray(Qxx, dtype=float).reshape(LX, LY)
    Qyx = np.asarray(Qyx, dtype=float).reshape(LX, LY)
    with np.errstate(divide="ignore", invalid="ignore"):
        S = np.sqrt(Qxx * Qxx + Qyx * Qyx)
        nx = np.sqrt(.5 * (1 + Qxx / S))
        ny = np.sign(Qyx) * np.sqrt(.5 * (1 - Qxx / S))
    # ring of (x, y): (x-1,y) (x-1,y-1) (x,y-1) (x+1,y-1) (x+1,y) (x+1,y+1) (x,y+1) (x-1,y+1)
    ring = [(1, 0), (1, 1), (0, 1), (-1, 1), (-1, 0), (-1, -1), (0, -1), (1, -1), (1, 0)]
    w = np.zeros((LX, LY))
    for s0, s1 in zip(ring[:-1], ring[1:]):
        a0, a1 = np.roll(nx, s0, axis=(0, 1)), np.roll(ny, s0, axis=(0, 1))
        b0, b1 = np.roll(nx, s1, axis=(0, 1)), np.roll(ny, s1, axis=(0, 1))
        ang = np.arctan2(a0 * b1 - a1 * b0, a0 * b0 + a1 * b1)
        w += np.where(np.abs(ang) > .5 * np.pi, ang - np.sign(ang) * np.pi, ang)
    return w / (2 * np.pi)


def count_defects(w: np.ndarray, threshold: float = 0.4):
    """Number of 4-connected (periodic) same-sign clusters of |w| > threshold,
    for positive and negative charge."""
    LX, LY = w.shape
    seen = np.zeros(w.shape, dtype=bool)
    counts = {1: 0, -1: 0}
    for x in range(LX):
        for y in range(LY):
            if seen[x, y] or not abs(w[x, y]) > threshold:
                continue
            s = 1 if w[x, y] > 0 else -1
            counts[s] += 1
            stack = [(x, y)]
            seen[x, y] = True
            while stack:
                i, j = stack.pop()
                for ni, nj in (((i + 1) % LX, j), ((i - 1) % LX, j), (i, (j + 1) % LY), (i, (j - 1) % LY)):
                    if not seen[ni, nj] and s * w[ni, nj] > threshold:
                        seen[ni, nj] = True
                        stack.append((ni, nj))
    return counts[1], counts[-1]


def statistics(state: dict, LX: int, LY: int, rest: float = 0.0) -> dict:
    vx, vy = velocity(state["ff"], LX, LY, rest)
    om = vorticity(vx, vy)
    out = {"mean_u2": float(np.mean(vx * vx + vy * vy)),
           "enstrophy_density": float(0.5 * np.mean(om * om))}
    w = charge(state["QQxx"], state["QQyx"], LX, LY)
    out["defects_plus"], out["defects_minus"] = count_defects(w)
    if "phi" in state:
        mask = np.asarray(state["phi"]).reshape(LX, LY) > 0.5
        out["perimeter"] = perimeter_4(mask)
        out["phi_area"] = float(mask.sum())
        o = om[mask]
        out["enstrophy_density_phi"] = float(0.5 * np.mean(o * o)) if o.size else 0.0
    return out
