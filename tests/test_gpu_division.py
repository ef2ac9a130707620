"""LyotropicWithDivision on the GPU against the reference's own division model.

The reference (oracle/_ref, src/models/lyotropic-with-division.cpp) draws
its division and death masks with its RNG at the start of every Step(); the
GPU lattice gets the same masks through mass_lb_set_phi_source as the rate
r = alpha*division_mask - beta*death_mask, and the conserve_phi correction
through mass_lb_set_phi_conservation when the model switches it on.
FP64: bit-identical fields after every run (periodic, walls, conservation).
FP32 fused: within the FP32 tolerances of tests/test_gpu_fp32.py against the
FP64 path with the same masks.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import LYO_C1, bits_equal, ff_dev, rel_l2

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402

DIV = {"alpha": 0.05, "beta": 0.03, "division-rate": 0.05, "division-time": 3,
       "division-radius": 4, "death-rate": 0.02, "death-time": 4, "death-radius": 3,
       "phi-critical": 1.2}
STATE = ("ff", "QQxx", "QQyx", "phi")


def params(**over):
    p = dict(LYO_C1)
    p.update(DIV)
    p.update({"config": "circle", "radius": 10, "conc": 1.0, "noise": 0.5})
    p.update(over)
    return p


def run_pair(p, LX, LY, bc, steps, precision=M.FP64, seed=11):
    ref = O.RefOracle(O.LYOTROPIC, p, LX, LY, bc, division=True)
    ref.configure(seed)
    lat = M.Lattice(M.LYOTROPIC, p, LX, LY, bc, precision)
    lat.upload_state({n: ref.get(n) for n in STATE})
    if ref.value("conserve_phi"):
        lat.set_phi_conservation(True, ref.value("totalphi"))
    prev = None
    masked = 0
    for _ in range(steps):
        ref.step(1)
        dm = ref.mask("division_mask").astype(np.float64)
        dd = ref.mask("death_mask").astype(np.float64)
        masked += int(dm.sum() + dd.sum())
        rate = p["alpha"] * dm - p["beta"] * dd
        if prev is None or not np.array_equal(rate, prev):
            lat.set_phi_source(rate)
            prev = rate
        lat.step(1)
    return ref, lat, masked


@pytest.mark.parametrize("LX,LY,bc", [(40, 36, 0), (64, 64, 0), (36, 40, 3), (40, 36, 2)])
def test_fp64_division_bit_identical(LX, LY, bc):
    ref, lat, masked = run_pair(params(), LX, LY, bc, 24)
    assert masked > 0, "the masks never switched on"
    assert ref.value("conserve_phi") == 0.0
    for n in STATE:
        assert bits_equal(lat.get(n), ref.get(n)), n
    lat.close()


@pytest.mark.parametrize("bc", [0, 1])
def test_fp64_conserve_phi_bit_identical(bc):
    p = params(alpha=0.0, beta=0.0)
    ref, lat, _ = run_pair(p, 40, 36, bc, 20)
    assert ref.value("conserve_phi") == 1.0
    for n in STATE:
        assert bits_equal(lat.get(n), ref.get(n)), n
    # the correction keeps the total at its configured value
    assert abs(lat.get("phi").sum() - ref.value("totalphi")) < 1e-9 * ref.value("totalphi")
    lat.close()


def test_fp32_fused_division_within_tolerance():
    p = params()
    LX = LY = 64
    ref = O.RefOracle(O.LYOTROPIC, p, LX, LY, 0, division=True)
    ref.configure(5)
    st = {n: ref.get(n) for n in STATE}
    a = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, M.FP32)
    b = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, M.FP64)
    assert a.uses_fused
    a.upload_state(st)
    b.upload_state(st)
    masked = 0
    for _ in range(10):
        ref.step(1)
        dm = ref.mask("division_mask").astype(np.float64)
        dd = ref.mask("death_mask").astype(np.float64)
        masked += int(dm.sum() + dd.sum())
        rate = p["alpha"] * dm - p["beta"] * dd
        a.set_phi_source(rate)
        b.set_phi_source(rate)
        a.step(1)
        b.step(1)
    assert masked > 0
    assert a.tile()[0] == 32                  # the source runs in the warp-strip kernel
    for n in STATE:
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x, 40.0), ff_dev(y, 40.0)
        assert rel_l2(x, y) < 1e-4, n
    # the source changed phi compared with no source at all
    c = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, M.FP32)
    c.upload_state(st)
    c.step(10)
    assert rel_l2(c.get("phi"), a.get("phi")) > 1e-4
    for lat in (a, b, c):
        lat.close()


def test_conserve_phi_moves_a_fused_lattice_to_the_sweeps():
    """conserve_phi needs a lattice-wide phi sum inside each sub-step, which
    the one-launch fused step has not: switching it on hands the FP32 state
    to the unfused sweeps, which hold phi at the given total."""
    p = params(alpha=0.0, beta=0.0)
    st = O.synthetic_state(O.LYOTROPIC, 64, 64, seed=12, flow=0.01)
    a = M.Lattice(M.LYOTROPIC, p, 64, 64, 0, M.FP32)
    assert a.uses_fused
    a.upload_state(st)
    a.step(2)
    total = float(a.get("phi").sum())
    a.set_phi_conservation(True, total)
    assert not a.uses_fused
    a.step(20)
    assert abs(a.get("phi").sum() - total) < 1e-4 * total
    a.close()


def test_unsupported_combinations_are_rejected():
    p = params()
    n = M.Lattice(M.NEMATIC, {"Gamma": 0.3, "xi": 0.7, "tau": 1.5, "CC": 0.1, "LL": 0.05},
                  64, 64, 0, M.FP64)
    with pytest.raises(M.MassLBError):
        n.set_phi_source(np.zeros(64 * 64))
    ens = M.Ensemble(M.LYOTROPIC, [LYO_C1], [(64, 64)])
    ens.runs[0].upload_state({"ff": np.tile(O.W_EQ * 40.0, (64 * 64, 1)), "QQxx": np.zeros(4096),
                              "QQyx": np.zeros(4096), "phi": np.full(4096, 0.5)})
    ens.runs[0].set_phi_source(np.full(64 * 64, 0.01))
    with pytest.raises(M.MassLBError):
        ens.step(1)
    with pytest.raises(M.MassLBError):
        ens.runs[0].set_phi_conservation(True, 1.0)
    ens.runs[0].set_phi_source(None)
    ens.step(1)
    for x in (n, ens):
        x.close()


def masks_rule(phi, LX, LY, draws, coef, phi_critical, radius, division):
    """The reference's SetMasks rule (src/models/lyotropic-with-division.cpp:
    35-106) restated for tests: candidates phi >= .5 in site order, one draw
    each, centre when draw < threshold, every site within the periodic
    circle test of a centre masked."""
    cand = np.flatnonzero(phi >= 0.5)
    p = phi[cand]
    thr = coef * p * (1 - p / phi_critical) if division else coef * p
    centers = cand[draws < thr]
    r2 = np.ceil(radius * radius)
    x = np.arange(LX)[:, None]
    y = np.arange(LY)[None, :]
    mask = np.zeros((LX, LY), dtype=bool)
    for c in centers:
        cx, cy = divmod(int(c), LY)
        dx = np.abs(x - cx)
        dx = np.minimum(dx % LX, LX - dx % LX)
        dy = np.abs(y - cy)
        dy = np.minimum(dy % LY, LY - dy % LY)
        mask |= (dx.astype(float) ** 2 + dy.astype(float) ** 2) <= r2
    return mask.reshape(-1), len(centers)


@pytest.mark.parametrize("LX,LY,bc,prec", [(40, 36, 0, M.FP64), (36, 40, 3, M.FP64),
                                           (64, 64, 0, M.FP32), (40, 36, 2, M.FP32)])
def test_device_masks_follow_reference_rule(LX, LY, bc, prec):
    """mass_lb_mask_candidates / mass_lb_draw_mask against the reference's
    rule on a phi with many candidates: masks, and the source they set
    (a lattice stepped with the device masks equals one stepped with
    mass_lb_set_phi_source(alpha*dm - beta*dd) bit for bit)."""
    rng = np.random.default_rng(LX + bc)
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=3, flow=0.01, phi_kind="disk",
                           radius=LX / 3)
    a = M.Lattice(M.LYOTROPIC, params(), LX, LY, bc, prec)
    b = M.Lattice(M.LYOTROPIC, params(), LX, LY, bc, prec)
    a.upload_state(st)
    b.upload_state(st)
    phi = a.get("phi")
    n = a.mask_candidates()
    assert n == int((phi >= 0.5).sum()) and n > 50
    expect = {}
    for kind, coef, radius in ((0, 0.3, 2.2), (1, 0.2, 0.0), (0, 0.05, 7.5), (1, 0.4, 1.0)):
        draws = rng.uniform(0, 1, n)
        a.draw_mask(kind, draws, coef, 1.3, radius, 0.05, 0.03)
        want, ncent = masks_rule(phi, LX, LY, draws, coef, 1.3, radius, kind == 0)
        assert ncent > 0
        assert np.array_equal(a.get_mask(kind), want), (kind, radius)
        expect[kind] = want
    rate = 0.05 * expect[0].astype(float) - 0.03 * expect[1].astype(float)
    b.set_phi_source(rate)
    a.step(3)
    b.step(3)
    for n_ in STATE:
        assert bits_equal(a.get(n_), b.get(n_)), n_
    with pytest.raises(M.MassLBError):
        a.draw_mask(0, np.zeros(n + 1), 0.1, 1.3, 1.0, 0.05, 0.03)
    with pytest.raises(M.MassLBError):
        a.draw_mask(2, np.zeros(n), 0.1, 1.3, 1.0, 0.05, 0.03)
    a.close()
    b.close()


@pytest.mark.parametrize("staged", [False, True])
@pytest.mark.parametrize("prec", [M.FP64, M.FP32])
def test_queued_masks_equal_direct_masks(prec, staged):
    """mass_lb_draw_masks_queued takes the same uniforms in the same order as
    mass_lb_draw_mask: over a run whose masks are redrawn on a schedule
    (division alone, death alone, both in one step), two lattices, one fed
    through the queue and one draw by draw, keep bit-identical masks and
    states, and the queue reports every draw it consumed. staged: the
    uniforms go up from the library's pinned staging buffer."""
    LX, LY = 64, 64
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=12, flow=0.01, phi_kind="disk",
                           radius=LX / 3)
    p = params()
    a = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, prec)
    b = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, prec)
    a.upload_state(st)
    b.upload_state(st)
    rng = np.random.default_rng(3)
    stream = rng.uniform(0, 1, 200000)
    pos_b = 0
    a.mask_supply(stream[:2 * LX * LY], staged)
    supplied = 2 * LX * LY
    for t in range(12):
        # the coefficients change half-way
        dc, dr, ec, er = (0.3, 2.5, 0.2, 1.5) if t < 6 else (0.45, 1.5, 0.1, 2.0)
        args = dict(division_coef=dc, division_radius=dr, death_coef=ec, death_radius=er,
                    phi_critical=1.3, alpha=0.05, beta=0.03)
        kinds = (1 if t % 3 == 0 else 0) | (2 if t % 2 == 0 else 0)
        if kinds:
            consumed = a.mask_consumed()
            assert consumed == pos_b
            if supplied - consumed < 2 * LX * LY:
                n = consumed + 2 * LX * LY - supplied
                a.mask_supply(stream[supplied:supplied + n], staged)
                supplied += n
            a.draw_masks_queued(kinds, **args)
            n = b.mask_candidates()
            if kinds & 1:
                b.draw_mask(0, stream[pos_b:pos_b + n], dc, 1.3, dr, 0.05, 0.03)
                pos_b += n
            if kinds & 2:
                b.draw_mask(1, stream[pos_b:pos_b + n], ec, 1.3, er, 0.05, 0.03)
                pos_b += n
        a.step(1)
        b.step(1)
    assert a.mask_consumed() == pos_b
    for kind in (0, 1):
        assert np.array_equal(a.get_mask(kind), b.get_mask(kind))
    for n_ in STATE:
        assert bits_equal(a.get(n_), b.get(n_)), n_
    # a queue that runs dry is reported
    c = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, prec)
    c.upload_state(st)
    c.mask_supply(stream[:10])
    c.draw_masks_queued(1, 0.3, 2.5, 0.2, 1.5, 1.3, 0.05, 0.03)
    with pytest.raises(M.MassLBError):
        c.mask_consumed()
    for x in (a, b, c):
        x.close()


@pytest.mark.parametrize("prec", [M.FP64, M.FP32])
def test_queued_masks_running_ahead(prec):
    """The plugin's supply policy: the host reads the consumed count of the
    draws the device has finished (mass_lb_mask_progress, no wait) and keeps
    2*LX*LY draws per draw in flight plus one more ahead, from the staging
    buffer. Masks and states stay bit-identical to draw-by-draw masks, the
    progress count never runs ahead of the true count, and it catches up
    once the device is idle."""
    LX, LY = 48, 40
    N = LX * LY
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=21, flow=0.01, phi_kind="disk",
                           radius=LX / 3)
    p = params()
    a = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, prec)
    b = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, prec)
    a.upload_state(st)
    b.upload_state(st)
    stream = np.random.default_rng(5).uniform(0, 1, 40 * N)
    supplied = pos_b = 0
    for t in range(18):
        kinds = (1 if t % 3 == 0 else 0) | (2 if t % 2 == 0 else 0)
        if kinds:
            consumed, pending = a.mask_progress()
            assert 0 <= pending <= 4 and consumed <= pos_b
            if pending > 2:
                consumed, pending = a.mask_consumed(), 0
            want = consumed + 2 * N * (pending + 1)
            if supplied < want:
                a.mask_supply(stream[supplied:want], True)
                supplied = want
            a.draw_masks_queued(kinds, 0.3, 2.5, 0.2, 1.5, 1.3, 0.05, 0.03)
            n = b.mask_candidates()
            if kinds & 1:
                b.draw_mask(0, stream[pos_b:pos_b + n], 0.3, 1.3, 2.5, 0.05, 0.03)
                pos_b += n
            if kinds & 2:
                b.draw_mask(1, stream[pos_b:pos_b + n], 0.2, 1.3, 1.5, 0.05, 0.03)
                pos_b += n
        a.step(1)
        b.step(1)
    a.synchronize()
    assert a.mask_progress() == (pos_b, 0)
    assert a.mask_consumed() == pos_b
    for kind in (0, 1):
        assert np.array_equal(a.get_mask(kind), b.get_mask(kind))
    for n_ in STATE:
        assert bits_equal(a.get(n_), b.get(n_)), n_
    a.close()
    b.close()


def test_queued_circles_wrapping_the_lattice():
    """Circles wider than half the lattice: the queued draw (each site looks
    for centres around it) marks the same sites as the direct draw (each
    centre writes its circle), both wrapping periodically."""
    LX, LY = 16, 12
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=4, flow=0.01, phi_kind="disk", radius=5)
    p = params()
    a = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, M.FP64)
    b = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, M.FP64)
    a.upload_state(st)
    b.upload_state(st)
    u = np.random.default_rng(8).uniform(0, 1, 64 * LX * LY)
    a.mask_supply(u[:6 * LX * LY])
    pos = 0
    for radius in (6.5, 4.2, 0.0):
        a.draw_masks_queued(3, 0.9, radius, 0.8, radius / 2, 1.3, 0.05, 0.03)
        n = b.mask_candidates()
        b.draw_mask(0, u[pos:pos + n], 0.9, 1.3, radius, 0.05, 0.03)
        b.draw_mask(1, u[pos + n:pos + 2 * n], 0.8, 1.3, radius / 2, 0.05, 0.03)
        pos += 2 * n
        for kind in (0, 1):
            assert np.array_equal(a.get_mask(kind), b.get_mask(kind)), (radius, kind)
        if radius > 6:
            assert a.get_mask(0).any()
    a.step(1)
    b.step(1)
    assert bits_equal(a.get("phi"), b.get("phi"))
    a.close()
    b.close()


@pytest.mark.parametrize("prec", [M.FP64, M.FP32])
def test_queued_masks_on_a_large_lattice(prec):
    """More than 1024 chunks of 1024 sites: every block of the queued draw
    walks several chunks and forms chunk offsets across segments of the
    count array. Masks and queue count equal the draw-by-draw path's."""
    LX, LY = 1100, 1000
    N = LX * LY
    st = O.synthetic_state(O.LYOTROPIC, LX, LY, seed=6, flow=0.01, phi_kind="disk",
                           radius=450)
    p = params()
    a = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, prec)
    b = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, prec)
    a.upload_state(st)
    b.upload_state(st)
    u = np.random.default_rng(11).uniform(0, 1, 4 * N)
    a.mask_supply(u[:4 * N], True)
    a.draw_masks_queued(3, 0.02, 3.0, 0.01, 2.0, 1.3, 0.05, 0.03)
    n = b.mask_candidates()
    assert n > N // 2
    b.draw_mask(0, u[:n], 0.02, 1.3, 3.0, 0.05, 0.03)
    b.draw_mask(1, u[n:2 * n], 0.01, 1.3, 2.0, 0.05, 0.03)
    assert a.mask_consumed() == 2 * n
    for kind in (0, 1):
        m = a.get_mask(kind)
        assert m.any() and np.array_equal(m, b.get_mask(kind)), kind
    a.step(1)
    b.step(1)
    assert bits_equal(a.get("phi"), b.get("phi"))
    a.close()
    b.close()
