"""Parity at the sizes the targets are stated on.

* Lyotropic FP64 at 256^2 (the CPU-runnable configuration: random director
  with S = 1, phi a tanh disk of radius 64, 100 steps): every field
  bit-identical to the reference's own OpenMP build run on the same state
  (the target is <= 1e-10 relative L2 per field; the test asserts equality
  and checks the bound as well).
* Lyotropic FP32 at 4096^2 (the throughput workload): after 10 steps within
  the FP32 tolerance of the FP64 mode on the same state, and over 200 steps
  the population total conserved and the state finite.
* Nematic at 2048^2 (the FP32-vs-FP64 configuration): FP32 within 1e-5
  relative L2 of FP64 per field after 100 steps.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_C1, NEM_C2, bits_equal, ff_dev, rel_l2

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_fp64_256_config_100_steps_equals_reference():
    LX = LY = 256
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=2024, radius=64)
    ref = O.RefOracle(O.LYOTROPIC, LYO_C1, LX, LY, 0)
    for k, v in st.items():
        ref.set(k, v)
    ref.step(100, os.cpu_count() or 1)
    lat = M.Lattice(M.LYOTROPIC, LYO_C1, LX, LY, 0, M.FP64)
    lat.upload_state(st)
    lat.step(100)
    for n in ("ff", "QQxx", "QQyx", "phi", "n", "ux", "uy", "MU", "HHxx", "sigmaXX",
              "sigmaXY", "sigma_bulk", "sigma_active_xx"):
        got, want = lat.get(n), ref.get(n)
        assert rel_l2(got, want) <= 1e-10, n
        assert bits_equal(got, want), n
    lat.close()


def test_fp32_4096_workload_against_fp64_and_conserved():
    L = 4096
    st = O.synthetic_state(O.LYOTROPIC, L, L, seed=1, radius=L / 4)
    a = M.Lattice(M.LYOTROPIC, LYO_C1, L, L, 0, M.FP32)
    b = M.Lattice(M.LYOTROPIC, LYO_C1, L, L, 0, M.FP64)
    a.upload_state(st)
    b.upload_state(st)
    del st
    a.step(10)
    b.step(10)
    for n in ("ff", "QQxx", "QQyx", "phi"):
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x), ff_dev(y)
        assert rel_l2(x, y) < 1e-4, n
    b.close()
    ftot, ptot = a.initial_totals()
    a.step(190)
    f, p, bad = a.checks()
    assert not bad
    assert abs(f - ftot) < 1e-7 * ftot
    assert abs(p - ptot) < 1e-5 * ptot
    a.close()


def test_nematic_2048_fp32_vs_fp64_100_steps():
    L = 2048
    st = O.synthetic_state(O.NEMATIC, L, L, seed=7)
    a = M.Lattice(M.NEMATIC, NEM_C2, L, L, 0, M.FP32)
    b = M.Lattice(M.NEMATIC, NEM_C2, L, L, 0, M.FP64)
    a.upload_state(st)
    b.upload_state(st)
    a.step(100)
    b.step(100)
    for n in ("ff", "QQxx", "QQyx"):
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x), ff_dev(y)
        assert rel_l2(x, y) < 1e-5, n
    a.close()
    b.close()
