"""Host logic of the surrogate's convolution entry points, no GPU needed.

The strip height (mass_sg_conv_strip_rows): each CTA of the forward /
input-gradient kernel marches down strips of that many output rows of one
image half, so the height must divide H, stay within 16, and balance the
strips over the SMs. And the argument checks of mass_sg_conv3x3 and
mass_sg_conv3x3_profile, which reject bad shapes, modes and missing
buffers before any device work."""
import ctypes
import math

import pytest

import mass_hd_b200 as M


def strip_rows(B, H, W, nsm):
    lib = ctypes.CDLL(M.library_path())
    f = lib.mass_sg_conv_strip_rows
    f.argtypes = [ctypes.c_int] * 4
    f.restype = ctypes.c_int
    return f(B, H, W, nsm)


def model(B, H, W, nsm):
    """The rule restated: minimise the busiest CTA's rows times the fitted
    cost of a row, 0.724 + 0.245 (R + 2) / R; ties go to the taller strip."""
    best, best_cost = 1, None
    for r in range(1, min(16, H) + 1):
        if H % r:
            continue
        items = B * (W // 128) * (H // r)
        cost = math.ceil(items / nsm) * r * (0.724 + 0.245 * (r + 2) / r)
        if best_cost is None or cost <= best_cost:
            best, best_cost = r, cost
    return best


def test_training_shapes():
    # 32 x 256^2: 1024 strips of 16 rows over 148 SMs (112 rows per CTA);
    # 16 x 256^2: 8-row strips give 56 rows per CTA against 64 with 16
    assert strip_rows(32, 256, 256, 148) == 16
    assert strip_rows(16, 256, 256, 148) == 8


@pytest.mark.parametrize("B,H,W,nsm", [(1, 1, 256, 148), (2, 3, 128, 148), (1, 5, 384, 148),
                                       (8, 24, 256, 148), (4, 32, 256, 148), (40, 128, 128, 148),
                                       (64, 1152, 1152, 148), (8, 256, 256, 132), (3, 97, 512, 148)])
def test_divides_height_and_follows_the_rule(B, H, W, nsm):
    r = strip_rows(B, H, W, nsm)
    assert 1 <= r <= 16 and H % r == 0
    assert r == model(B, H, W, nsm)


def test_degenerate_arguments_fall_back_to_one_row():
    assert strip_rows(0, 256, 256, 148) == 1
    assert strip_rows(4, 256, 64, 148) == 1
    assert strip_rows(4, 256, 256, 0) == 1


def _conv_fn(name):
    lib = ctypes.CDLL(M.library_path())
    f = getattr(lib, name)
    vp, i = ctypes.c_void_p, ctypes.c_int
    f.argtypes = [vp, vp, i, i, i, i, i] + [vp] * 8 + ([vp, vp] if name.endswith("profile") else []) + [vp]
    f.restype = ctypes.c_int
    return f


# Argument checks run on the host before any device work, so they can be
# exercised without a GPU: fake non-null pointers never reach a kernel.
P = ctypes.c_void_p(64)


@pytest.mark.parametrize("name", ["mass_sg_conv3x3", "mass_sg_conv3x3_profile"])
@pytest.mark.parametrize("nout,mode,B,H,W,why", [
    (64, 1, 1, 8, 100, "W not a multiple of 128"),
    (64, 1, 0, 8, 128, "no image"),
    (64, 9, 1, 8, 128, "unknown mode"),
    (16, 1, 1, 8, 128, "nout 16 outside the output layer"),
    (64, 3, 1, 8, 128, "the output layer with nout 64"),
])
def test_convolution_rejects_bad_arguments(name, nout, mode, B, H, W, why):
    f = _conv_fn(name)
    extra = [P, P] if name.endswith("profile") else []
    r = f(P, P, nout, mode, B, H, W, P, P, P, P, P, P, P, P, *extra, None)
    assert r < 0, why


def test_profile_needs_its_counter_buffers():
    f = _conv_fn("mass_sg_conv3x3_profile")
    assert f(P, P, 64, 1, 1, 8, 128, P, P, P, P, P, P, P, P, None, P, None) < 0
    assert f(P, P, 64, 1, 1, 8, 128, P, P, P, P, P, P, P, P, P, None, None) < 0
