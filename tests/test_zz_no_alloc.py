"""The allocation-free conservation sums (mass_lb_state_sums_noalloc).

Callers that cannot allocate device memory - a program whose HBM another
allocator owns in full, or a monitoring path that must not pay cudaMalloc's
synchronization - get the sums of mass_lb_checks from this entry point,
whose scratch is a fixed array inside the library. This test calls it
through the C ABI on the state of a live lattice, twice in a row (the array
keeps the previous call's contents), and compares it with mass_lb_checks on
the same lattice. It also checks that a lattice above the 8192^2 limit is
refused before any device work. It runs alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_ALL, NEM_ALL

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402

REL = 1e-12   # both reductions are compensated FP64 sums of the same values


def noalloc_fn():
    lib = M.load_library()
    f = lib.mass_lb_state_sums_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_uint, C.c_uint, C.c_double,
                  C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                  C.POINTER(C.c_int)]
    return f


def call(f, lat, rho=40.0):
    planes, stride, n = lat.device_state()
    fs, ps, bad = C.c_double(), C.c_double(), C.c_int()
    r = f(planes, stride, n, lat.LX, lat.LY, rho, lat.stream, C.byref(fs), C.byref(ps),
          C.byref(bad))
    assert r == 0, M.load_library().mass_lb_last_error()
    return fs.value, ps.value, bool(bad.value)


@pytest.mark.parametrize("model,params,L", [(O.LYOTROPIC, LYO_ALL, 256), (O.NEMATIC, NEM_ALL, 192)])
def test_noalloc_sums_match_checks_twice(model, params, L):
    f = noalloc_fn()
    st = O.synthetic_state(model, L, L, seed=41, flow=0.01)
    lat = M.Lattice(model, params, L, L, 0, M.FP32)
    assert lat.uses_fused
    lat.upload_state(st)
    lat.step(4)
    want_f, want_p, want_bad = lat.checks()
    for _ in range(2):
        got_f, got_p, got_bad = call(f, lat)
        assert got_f == pytest.approx(want_f, rel=REL)
        if model == O.LYOTROPIC:
            assert got_p == pytest.approx(want_p, rel=REL)
        else:
            assert got_p == 0.0
        assert got_bad == want_bad is False
    # a later step changes the state; the static scratch must not carry over
    lat.step(1)
    want_f, want_p, _ = lat.checks()
    got_f, got_p, _ = call(f, lat)
    assert got_f == pytest.approx(want_f, rel=REL)
    assert got_p == pytest.approx(want_p, rel=REL)
    lat.close()


def test_noalloc_flags_nonfinite_like_checks():
    f = noalloc_fn()
    st = O.synthetic_state(O.LYOTROPIC, 128, 128, seed=3)
    st["phi"] = st["phi"].copy()
    st["phi"][1234] = np.inf
    lat = M.Lattice(O.LYOTROPIC, LYO_ALL, 128, 128, 0, M.FP32)
    lat.upload_state(st)
    assert lat.checks()[2] is True
    assert call(f, lat)[2] is True
    lat.close()


def test_noalloc_rejects_lattices_above_the_limit():
    f = noalloc_fn()
    lat = M.Lattice(O.NEMATIC, NEM_ALL, 128, 128, 0, M.FP32)
    planes, stride, n = lat.device_state()
    fs, ps, bad = C.c_double(), C.c_double(), C.c_int()
    r = f(planes, 8192 * 8193, n, 8192, 8193, 40.0, lat.stream, C.byref(fs), C.byref(ps),
          C.byref(bad))
    assert r == -1
    assert b"limit of the static scratch" in M.load_library().mass_lb_last_error()
    lat.close()


def test_noalloc_rejects_host_planes():
    """Planes that are not device memory of the current device are refused
    before any launch."""
    f = noalloc_fn()
    host = np.zeros(12 * 64 * 64, dtype=np.float32)
    fs, ps, bad = C.c_double(), C.c_double(), C.c_int()
    r = f(host.ctypes.data, 64 * 64, 12, 64, 64, 40.0, None, C.byref(fs), C.byref(ps),
          C.byref(bad))
    assert r == -1
    assert b"not device memory" in M.load_library().mass_lb_last_error()
