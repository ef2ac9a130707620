"""Shared test helpers (parameter sets, comparisons, golden loading)."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# physics of the 256^2 CPU-runnable lyotropic configuration (CN->CC,
# Aphi->AA, Kphi->KK, Kn->LL, Gammaphi->GammaP, tau -> tauNem = tauIso)
LYO_C1 = dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5, tauIso=1.5, rho=40.0,
              friction=0.0, AA=0.1, CC=0.1, LL=0.05, KK=0.05, zeta=0.01,
              zetaI=0.0, conc=1.0, npc=1)
# every term switched on
LYO_ALL = dict(GammaQ=0.3, GammaP=0.1, xi=0.7, tauNem=1.5, tauIso=1.2, rho=40.0,
               friction=0.02, AA=0.1, CC=0.1, LL=0.05, KK=0.05, zeta=0.03,
               zetaI=0.01, conc=0.9, npc=1)
# physics of the 2048^2 nematic FP32-vs-FP64 configuration (CC fixed at 0.1)
NEM_C2 = dict(Gamma=0.3, xi=0.7, tau=1.5, rho=40.0, friction=0.0, CC=0.1,
              LL=0.05, zeta=0.02, npc=1)
NEM_ALL = dict(NEM_C2, friction=0.01)

W_EQ = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "*_bc*.npz")))


def load_golden(path):
    z = np.load(path)
    return json.loads(str(z["meta"])), z


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    return num / den if den > 0 else num


def ff_dev(ff, rho=40.0):
    """Populations minus their rest-state part t_v*rho."""
    return np.asarray(ff).reshape(-1, 9) - W_EQ[None, :] * rho


def bits_equal(a, b):
    """Bit-for-bit equality of two float64 arrays (distinguishes -0 from +0,
    which np.array_equal does not)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
