"""Batched ensemble (mass_lb_ensemble_*) against the single-lattice fused path.

Each run of an ensemble must end bit-identical to the same run stepped on
its own: the ensemble kernel executes the same per-site arithmetic with the
same FP32 parameters, only the work distribution differs. Covered: uneven
sizes (square and not, LY not a multiple of the 56-column strip), per-run
parameters, odd and even step counts (graph pairs plus a single launch),
several chunk heights, the diagnostic fields and statistics of a run after
ensemble steps, and argument validation.
"""
import numpy as np
import pytest

import mass_hd_b200 as M
from mass_hd_b200.ensemble_case import sweep
from mass_hd_b200.run_case import PARAMS, REST

pytestmark = pytest.mark.gpu

FIELDS = ("ff", "QQxx", "QQyx", "phi")


def uneven_cases(seed=3):
    rng = np.random.default_rng(seed)
    sizes = [(128, 128), (64, 192), (200, 68), (96, 100), (256, 64), (72, 120)]
    out = []
    for LX, LY in sizes:
        p = dict(PARAMS["lyotropic"])
        p["zeta"] = float(rng.uniform(0.002, 0.04))
        p["LL"] = float(rng.uniform(0.02, 0.08))
        p["xi"] = float(rng.choice([0.3, 0.7, 1.0]))
        theta = rng.uniform(0, np.pi, LX * LY)
        st = {"QQxx": np.cos(2 * theta), "QQyx": np.sin(2 * theta),
              "ff": np.tile(REST * 40.0, (LX * LY, 1)) + rng.normal(0, 0.05, (LX * LY, 9)),
              "phi": rng.normal(0.5, 0.05, LX * LY)}
        out.append((p, (LX, LY), st))
    return out


def singles(cases, steps, rows=64):
    out = []
    for p, (LX, LY), st in cases:
        lat = M.Lattice(M.LYOTROPIC, p, LX, LY, 0, M.FP32)
        lat.set_tile(32, min(rows, LX))
        lat.upload_state(st)
        lat.step(steps)
        out.append(lat)
    return out


@pytest.mark.parametrize("steps", [1, 4, 7])
def test_ensemble_matches_single_runs(steps):
    cases = uneven_cases()
    ens = M.Ensemble(M.LYOTROPIC, [c[0] for c in cases], [c[1] for c in cases])
    for run, (_, _, st) in zip(ens.runs, cases):
        run.upload_state(st)
    ens.step(steps)
    assert ens.rows in (32, 64, 128, 256)
    ref = singles(cases, steps)
    for i, (run, lat) in enumerate(zip(ens.runs, ref)):
        for n in FIELDS:
            a, b = run.get(n), lat.get(n)
            assert np.isfinite(a).all()
            assert np.array_equal(a, b), (i, n, float(np.abs(a - b).max()))
    ens.close()


@pytest.mark.parametrize("rows", ["32", "128"])
def test_chunk_height_does_not_change_results(monkeypatch, rows):
    monkeypatch.setenv("MASS_LB_ENSEMBLE_ROWS", rows)
    cases = uneven_cases(seed=5)[:4]
    ens = M.Ensemble(M.LYOTROPIC, [c[0] for c in cases], [c[1] for c in cases])
    for run, (_, _, st) in zip(ens.runs, cases):
        run.upload_state(st)
    ens.step(3)
    assert ens.rows == int(rows)
    ref = singles(cases, 3)
    for run, lat in zip(ens.runs, ref):
        for n in FIELDS:
            assert np.array_equal(run.get(n), lat.get(n)), n
    ens.close()


def test_steps_in_pieces_equal_one_call():
    cases = uneven_cases(seed=9)[:3]
    a = M.Ensemble(M.LYOTROPIC, [c[0] for c in cases], [c[1] for c in cases])
    b = M.Ensemble(M.LYOTROPIC, [c[0] for c in cases], [c[1] for c in cases])
    for ra, rb, (_, _, st) in zip(a.runs, b.runs, cases):
        ra.upload_state(st)
        rb.upload_state(st)
    a.step(6)
    for k in (1, 2, 3):
        b.step(k)
    for ra, rb in zip(a.runs, b.runs):
        for n in FIELDS:
            assert np.array_equal(ra.get(n), rb.get(n)), n
    a.close()
    b.close()


def test_run_diagnostics_and_statistics_after_ensemble_steps():
    cases = uneven_cases(seed=11)[:2]
    ens = M.Ensemble(M.LYOTROPIC, [c[0] for c in cases], [c[1] for c in cases])
    for run, (_, _, st) in zip(ens.runs, cases):
        run.upload_state(st)
    ens.step(5)
    ref = singles(cases, 5)
    for run, lat in zip(ens.runs, ref):
        for n in ("ux", "uy", "MU", "HHxx", "sigmaXY"):
            assert np.array_equal(run.get(n), lat.get(n)), n
        assert run.statistics() == lat.statistics()
        f, p = run.runtime_checks()
        ftot, ptot = run.initial_totals()
        assert abs(f - ftot) < 1e-2 * ftot and np.isfinite(p)
    ens.close()


def test_sweep_workload_sample_bit_identical():
    cases = sweep(8, seed=7, sizes=(128, 192, 256))
    ens = M.Ensemble(M.LYOTROPIC, [c[0] for c in cases], [c[1] for c in cases])
    for run, (_, _, st) in zip(ens.runs, cases):
        run.upload_state(st)
    ens.step(10)
    ref = singles(cases, 10)
    for run, lat in zip(ens.runs, ref):
        for n in FIELDS:
            assert np.array_equal(run.get(n), lat.get(n)), n
    ens.close()


def test_nematic_ensemble():
    rng = np.random.default_rng(2)
    sizes = [(128, 64), (64, 128), (100, 96)]
    params = []
    states = []
    for LX, LY in sizes:
        p = dict(PARAMS["nematic"])
        p["zeta"] = float(rng.uniform(0.005, 0.03))
        params.append(p)
        th = rng.uniform(0, np.pi, LX * LY)
        states.append({"QQxx": np.cos(2 * th), "QQyx": np.sin(2 * th),
                       "ff": np.tile(REST * 40.0, (LX * LY, 1))})
    ens = M.Ensemble(M.NEMATIC, params, sizes)
    for run, st in zip(ens.runs, states):
        run.upload_state(st)
    ens.step(5)
    for run, p, (LX, LY), st in zip(ens.runs, params, sizes, states):
        lat = M.Lattice(M.NEMATIC, p, LX, LY, 0, M.FP32)
        lat.set_tile(32, 64)
        lat.upload_state(st)
        lat.step(5)
        for n in ("ff", "QQxx", "QQyx"):
            assert np.array_equal(run.get(n), lat.get(n)), n
        lat.close()
    ens.close()


def test_ensemble_rejects_unsupported_runs():
    p = PARAMS["lyotropic"]
    with pytest.raises(M.MassLBError):
        M.Ensemble(M.LYOTROPIC, [p], [(64, 62)])          # LY % 4 != 0
    with pytest.raises(M.MassLBError):
        M.Ensemble(M.LYOTROPIC, [dict(p, npc=2)], [(64, 64)])
    with pytest.raises(M.MassLBError):
        M.Ensemble(M.LYOTROPIC, [p] * 193, [(64, 64)] * 193)
