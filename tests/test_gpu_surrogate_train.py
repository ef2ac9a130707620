"""The trained surrogate against the method without it, on the GPU.

A small version of the training workload (128^2 lattices, simulator-made
(t, t+50) pairs, a few hundred AdamW steps through the library's own
forward and backward kernels) must predict the held-out Q fields better
than persistence (the fields left as they are), which is what the plain
method's own state gives without running it. The hybrid controller is
checked at both ends of its threshold: with 0 every check rejects the
surrogate and the runs must end bit-identical to plain LB stepping; with
an unbounded threshold the surrogate takes every jump it is offered.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

import mass_hd_b200.surrogate as G  # noqa: E402
from mass_hd_b200 import lb  # noqa: E402

L = 128


@pytest.fixture(scope="module")
def trained():
    ntrain, nheld, npairs = 8, 2, 20
    fields, _ = G.generate_dataset(ntraj=ntrain + nheld, L=L, pairs=npairs, t_min=500,
                                   t_max=4500, seed=4)
    n_train = ntrain * 2 * npairs
    mean, scale = G.normalise(fields[:n_train])
    fields[n_train:].sub_(torch.tensor(mean, device="cuda")).div_(torch.tensor(scale, device="cuda"))
    P = G.Params(seed=2)
    P.mean, P.scale = mean, scale
    losses = G.train(P, fields, G.pair_indices(ntrain, npairs), epochs=25, batch=16, lr=1e-3)
    ev = G.evaluate(P, fields, G.pair_indices(nheld, npairs) + n_train, batch=8)
    return P, losses, ev


def test_training_beats_persistence_on_held_out_runs(trained):
    _, losses, ev = trained
    assert losses[-1] < losses[0]
    s, p = ev["surrogate_mse"], ev["persistence_mse"]
    print("held-out mse surrogate", s, "persistence", p)
    for c in (0, 1):                                  # Qxx, Qyx
        assert s[c] < p[c], (c, s[c], p[c])


def _ensemble(n=2, seed=9):
    rng = np.random.default_rng(seed)
    zetas = rng.uniform(0.005, 0.03, n)
    states = [G.initial_state(L, rng) for _ in range(n)]
    ens = lb.Ensemble(lb.LYOTROPIC, [G.training_params(z) for z in zetas], [(L, L)] * n)
    for run, st in zip(ens.runs, states):
        run.upload_state(st)
    ens.step(500)
    return ens


def test_hybrid_with_zero_threshold_is_plain_lb(trained):
    P = trained[0]
    a, b = _ensemble(), _ensemble()
    res = G.hybrid(P, a, 1000, jump=50, M=10, threshold=0.0)
    b.step(1000)
    assert res["surrogate_jumps"] == 0 and res["plain_jumps_rejected"] == 18
    for ra, rb in zip(a.runs, b.runs):
        for n in ("ff", "QQxx", "QQyx", "phi"):
            assert np.array_equal(ra.get(n), rb.get(n)), n
    a.close()
    b.close()


def test_hybrid_with_open_threshold_uses_the_surrogate(trained):
    P = trained[0]
    ens = _ensemble()
    res = G.hybrid(P, ens, 1000, jump=50, M=10, threshold=float("inf"))
    assert res["surrogate_jumps"] == 18 and res["checks"] == 2
    for run in ens.runs:
        f, p, bad = run.checks()
        assert not bad and abs(f - 40.0 * L * L) < 1e-2 * 40.0 * L * L
    ens.close()
