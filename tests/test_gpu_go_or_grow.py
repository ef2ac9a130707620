"""GoOrGrow on the GPU against the reference's own go-or-grow model.

The reference (oracle/_ref, src/models/go-or-grow.cpp) is configured with its
own Configure() - initial circle, dry free-energy relaxation, rest-state
populations, phenotype noise smoothed over a correlation length - and the
GPU lattice gets that state (ff, QQxx, QQyx, phi, m). Every Step() the
reference draws its division/death masks; the GPU gets the growth rate
alpha*division_mask - beta*death_mask through mass_lb_set_phi_source.
FP64: every state field, chi and every derived field bit-identical after
the run, for the periodic lattice and all four wall types, both growth
rules (growTogether 0/1), and the conserve_phi branch. The device
relaxation (mass_lb_relax_free_energy) is checked the same way against a
reference configured with and without relaxation. FP32 (unfused sweeps):
within the FP32 tolerances against the FP64 path.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import bits_equal, ff_dev, rel_l2

pytestmark = pytest.mark.gpu

import mass_hd_b200 as M  # noqa: E402

# the shipped runcard's physics (test.dat of the reference's cases/), with
# the phenotype terms, activity and both division and death switched on
GOG = {"GammaQ": 0.3, "GammaP": 5e-2, "zeta": 0.02, "zetaI": 0.01, "friction": 0.01,
       "tauNem": 1.0, "tauIso": 1.2, "AA": 0.03, "CC": 0.1, "LL": 0.002, "KK": 0.06,
       "rho": 40.0, "xi": 0.3, "B": 0.1, "Snem": 1.0, "config": "circle", "level": 0,
       "radius": 9, "conc": 1.0, "noise": 1.0, "angle": 0, "npc": 1,
       "relax-steps": 40, "relax-dt": 1.0, "relax-phi": 1, "relax-Q": 1,
       "chi-config": "noise", "chi0": 0.6, "chi-noise": 0.05, "chi-length": 2,
       "Dchi": 0.005, "Achi": 0.1, "Ochi": 0.05, "phiswitch": 0.5, "growTogether": 0,
       "alpha": 0.002, "beta": 0.001, "division-rate": 0.1, "division-time": 2,
       "division-radius": 3, "death-rate": 0.02, "death-time": 3, "death-radius": 2,
       # below the circle's plateau, so that the crowding penalty B acts
       "phi-critical": 0.9}
STATE = ("ff", "QQxx", "QQyx", "phi", "m")
DERIVED = ("chi", "n", "ux", "uy", "ux_phi", "uy_phi", "HHxx", "HHyx", "MU", "dxQQxx",
           "dyQQxx", "dxQQyx", "dyQQyx", "sigmaXX", "sigmaYY", "sigmaYX", "sigmaXY",
           "sigma_bulk", "sigma_elastic_xx", "sigma_elastic_yx", "sigma_phase_field_xx",
           "sigma_phase_field_yx", "sigma_active_xx", "sigma_active_yx")


def params(**over):
    p = dict(GOG)
    p.update(over)
    return p


def rate_of(ref, p):
    dm = ref.mask("division_mask").astype(np.float64)
    dd = ref.mask("death_mask").astype(np.float64)
    return p["alpha"] * dm - p["beta"] * dd, int(dm.sum() + dd.sum())


def run_pair(p, LX, LY, bc, steps, precision=M.FP64, seed=17):
    ref = O.RefOracle(O.GO_OR_GROW, p, LX, LY, bc)
    ref.configure(seed)
    lat = M.Lattice(M.GO_OR_GROW, p, LX, LY, bc, precision)
    lat.upload_state({n: ref.get(n) for n in STATE})
    if ref.value("conserve_phi"):
        lat.set_phi_conservation(True, ref.value("totalphi"))
    prev, masked = None, 0
    for _ in range(steps):
        ref.step(1)
        rate, k = rate_of(ref, p)
        masked += k
        if prev is None or not np.array_equal(rate, prev):
            lat.set_phi_source(rate)
            prev = rate
        lat.step(1)
    return ref, lat, masked


@pytest.mark.parametrize("LX,LY,bc,grow", [(40, 36, 0, 0), (40, 36, 0, 1), (36, 40, 1, 0),
                                           (40, 36, 2, 1), (36, 40, 3, 0), (40, 36, 4, 1)])
def test_fp64_go_or_grow_bit_identical(LX, LY, bc, grow):
    p = params(growTogether=grow)
    ref, lat, masked = run_pair(p, LX, LY, bc, 16)
    assert masked > 0, "the masks never switched on"
    assert ref.value("conserve_phi") == 0.0
    for n in STATE + DERIVED:
        assert bits_equal(lat.get(n), ref.get(n)), n
    # the phenotype moved: chi is neither constant nor equal to its start
    chi = lat.get("chi")
    assert chi.std() > 1e-3
    lat.close()


def test_fp64_go_or_grow_conserve_phi():
    p = params(alpha=0.0, beta=0.0)
    ref, lat, _ = run_pair(p, 40, 36, 0, 16)
    assert ref.value("conserve_phi") == 1.0
    for n in STATE + ("chi",):
        assert bits_equal(lat.get(n), ref.get(n)), n
    lat.close()


def test_fp64_go_or_grow_predictor_fields():
    """mN, QNxx, phn: the step-internal values after the last corrector."""
    p = params(npc=2)
    ref, lat, _ = run_pair(p, 36, 36, 0, 6)
    for n in ("mN", "QNxx", "QNyx", "phn", "fn"):
        assert bits_equal(lat.get(n), ref.get(n)), n
    lat.close()


@pytest.mark.parametrize("bc,relax_phi,relax_Q", [(0, 1, 1), (0, 1, 0), (1, 1, 1),
                                                  (3, 0, 1), (4, 1, 1)])
def test_fp64_relaxation_bit_identical(bc, relax_phi, relax_Q):
    """mass_lb_relax_free_energy == GoOrGrow::RelaxFreeEnergy: the reference
    configured with relax-steps = 0 gives the unrelaxed state (the
    relaxation draws no random numbers), the one with relax-steps = 30 the
    relaxed state and totalphi."""
    LX, LY = 36, 40
    pr = params(**{"relax-steps": 30, "relax-phi": relax_phi, "relax-Q": relax_Q,
                   "relax-dt": 0.8})
    p0 = params(**{"relax-steps": 0})
    a = O.RefOracle(O.GO_OR_GROW, pr, LX, LY, bc)
    a.configure(5)
    b = O.RefOracle(O.GO_OR_GROW, p0, LX, LY, bc)
    b.configure(5)
    lat = M.Lattice(M.GO_OR_GROW, pr, LX, LY, bc, M.FP64)
    lat.upload_state({n: b.get(n) for n in ("ff", "QQxx", "QQyx", "phi")})
    total = lat.relax_free_energy(30, 0.8, relax_phi, relax_Q)
    for n in ("QQxx", "QQyx", "phi"):
        assert bits_equal(lat.get(n), a.get(n)), n
    assert total == a.value("totalphi")
    assert lat.initial_totals()[1] == total
    if relax_phi:
        assert not np.array_equal(a.get("phi"), b.get("phi"))
    lat.close()


def test_fp32_go_or_grow_within_tolerance():
    """The unfused FP32 sweeps (LY = 62 is not a multiple of 4, so the fused
    kernel does not take this lattice) against FP64, masks on."""
    p = params()
    LX, LY = 64, 62
    ref = O.RefOracle(O.GO_OR_GROW, p, LX, LY, 0)
    ref.configure(3)
    st = {n: ref.get(n) for n in STATE}
    a = M.Lattice(M.GO_OR_GROW, p, LX, LY, 0, M.FP32)
    b = M.Lattice(M.GO_OR_GROW, p, LX, LY, 0, M.FP64)
    assert not a.uses_fused
    a.upload_state(st)
    b.upload_state(st)
    for _ in range(20):
        ref.step(1)
        rate, _ = rate_of(ref, p)
        a.set_phi_source(rate)
        b.set_phi_source(rate)
        a.step(1)
        b.step(1)
    for n in STATE + ("chi",):
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x, 40.0), ff_dev(y, 40.0)
        assert rel_l2(x, y) < 1e-4, n
    a.close()
    b.close()


@pytest.mark.parametrize("bc", [1, 2, 3, 4])
def test_fp32_go_or_grow_walls_within_tolerance(bc):
    """The FP32 sweeps with every wall type against FP64, masks on."""
    p = params()
    LX, LY = 48, 40
    ref = O.RefOracle(O.GO_OR_GROW, p, LX, LY, bc)
    ref.configure(8)
    st = {n: ref.get(n) for n in STATE}
    a = M.Lattice(M.GO_OR_GROW, p, LX, LY, bc, M.FP32)
    b = M.Lattice(M.GO_OR_GROW, p, LX, LY, bc, M.FP64)
    a.upload_state(st)
    b.upload_state(st)
    for _ in range(12):
        ref.step(1)
        rate, _ = rate_of(ref, p)
        a.set_phi_source(rate)
        b.set_phi_source(rate)
        a.step(1)
        b.step(1)
    for n in STATE + ("chi",):
        x, y = a.get(n), b.get(n)
        if n == "ff":
            x, y = ff_dev(x, 40.0), ff_dev(y, 40.0)
        assert rel_l2(x, y) < 1e-4, (bc, n)
    a.close()
    b.close()


def test_fp32_conserve_phi_parallel_sum():
    """FP32 sweeps take countphi from a parallel FP64 sum (FP64 keeps the
    serial site order): with division and death off, phi stays at its
    configured total and the fields track the FP64 run."""
    p = params(alpha=0.0, beta=0.0)
    LX, LY = 96, 80
    ref = O.RefOracle(O.GO_OR_GROW, p, LX, LY, 0)
    ref.configure(4)
    assert ref.value("conserve_phi") == 1.0
    st = {n: ref.get(n) for n in STATE}
    total = ref.value("totalphi")
    a = M.Lattice(M.GO_OR_GROW, p, LX, LY, 0, M.FP32)
    b = M.Lattice(M.GO_OR_GROW, p, LX, LY, 0, M.FP64)
    for lat in (a, b):
        lat.upload_state(st)
        lat.set_phi_conservation(True, total)
        lat.step(40)
    assert abs(a.get("phi").sum() - total) < 1e-4 * total
    for n in ("phi", "m", "QQxx"):
        assert rel_l2(a.get(n), b.get(n)) < 1e-4, n
    a.close()
    b.close()


def test_go_or_grow_checkpoint_resumes_bit_identical(tmp_path):
    p = params()
    ref = O.RefOracle(O.GO_OR_GROW, p, 36, 36, 2)
    ref.configure(9)
    st = {n: ref.get(n) for n in STATE}
    rate = np.where(st["phi"] > 0.5, 0.002, 0.0)
    a = M.Lattice(M.GO_OR_GROW, p, 36, 36, 2, M.FP64)
    a.upload_state(st)
    a.set_phi_source(rate)
    a.step(5)
    path = os.path.join(tmp_path, "gog.ckpt")
    a.save(path)
    a.step(5)
    b = M.Lattice(M.GO_OR_GROW, p, 36, 36, 2, M.FP64)
    b.load(path)
    b.set_phi_source(rate)
    b.step(5)
    for n in STATE + ("chi",):
        assert np.array_equal(a.get(n), b.get(n)), n
    a.close()
    b.close()


def test_go_or_grow_rejections():
    p = params()
    lyo = M.Lattice(M.LYOTROPIC, p, 64, 64, 0, M.FP64)
    with pytest.raises(M.MassLBError):
        lyo.upload_field("m", np.zeros(64 * 64))
    with pytest.raises(M.MassLBError):
        lyo.get("chi")
    with pytest.raises(M.MassLBError):
        lyo.relax_free_energy(1)
    with pytest.raises(M.MassLBError):
        lyo.set_go_or_grow_params(p)
    with pytest.raises(M.MassLBError):
        M.Ensemble(M.GO_OR_GROW, [p], [(64, 64)])
    g32 = M.Lattice(M.GO_OR_GROW, p, 64, 64, 0, M.FP32)
    with pytest.raises(M.MassLBError):
        g32.get("mN")
    for x in (lyo, g32):
        x.close()


@pytest.mark.parametrize("change", ["relax", "params", "load"])
def test_go_or_grow_derived_fields_survive_state_changes(change, tmp_path):
    """On a periodic lattice the step leaves its derived fields (u, H, mu,
    the stresses) to be recomputed on demand. A relaxation, new phenotype
    parameters or a checkpoint load in between do not change them: they
    stay those of the step, as on a lattice that downloaded them first (the
    relaxation leaves its own H and mu, as it always has), and a loaded
    state is the saved one."""
    p = params()
    ref = O.RefOracle(O.GO_OR_GROW, p, 40, 36, 0)
    ref.configure(5)
    st = {n: ref.get(n) for n in STATE}
    rate = np.where(st["phi"] > 0.5, 0.002, 0.0)
    a = M.Lattice(M.GO_OR_GROW, p, 40, 36, 0, M.FP64)
    b = M.Lattice(M.GO_OR_GROW, p, 40, 36, 0, M.FP64)
    path = os.path.join(tmp_path, "gog.ckpt")
    for x in (a, b):
        x.upload_state(st)
        x.set_phi_source(rate)
        x.step(4)
    b.save(path)
    want = {n: a.get(n) for n in DERIVED if n != "chi"}
    if change == "relax":
        b.relax_free_energy(5, 1.0, True, True)
        for n in ("HHxx", "HHyx", "MU"):
            del want[n]
    elif change == "params":
        b.set_go_or_grow_params(params(B=0.5, Snem=0.8, **{"phi-critical": 0.7}))
    else:
        b.step(3)
        b.load(path)
        want = {n: a.get(n) for n in ("ff", "QQxx", "phi", "m")}
    for n, v in want.items():
        assert bits_equal(b.get(n), v), n
    a.close()
    b.close()
