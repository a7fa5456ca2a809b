"""What the learned proposal gains (marked gpu): on an 8F7 zeta delta
search, both the exhaustive sweep and the proposal start with the walk's
singularity filter; the sweep walks every survivor, the proposal walks only
the survivors its trained network ranks highest. At the same budget, the
network's choice finds more of the sweep's top-20 deltas than the same
number of survivors chosen at random (the method without the network), and
every delta it reports is the sweep's own value for that candidate. The
network's target is membership of the training walks' top 1% of deltas,
its features the counts of x and y components by magnitude."""
import numpy as np
import pytest

from cmfw import mlp as cm
from cmfw import proposal as prop

pytestmark = pytest.mark.gpu


def test_trained_proposal_beats_the_same_budget_without_it(cuda):
    S = prop.DeltaSearch(8, 7, 0, 4, 1000, 50, "df64", seed=777, batch=1 << 20)
    n, frac, k = 1 << 23, 0.1, 20
    truth, deltas, n_valid, _, st = S.sweep(n, k)
    assert len(truth) == k and n_valid > 1000 and st["survivors"] >= n_valid
    data = S.training_set(1 << 25, 1 << 40)
    net = cm.Mlp(1 << 16, seed=1)
    S.train(net, data[:4], epochs=30)
    p_idx, p_d, n_walk, _, stp = S.propose(net, n, frac, k)
    assert abs(n_walk - frac * st["survivors"]) <= 1 + 0.01 * n_walk
    r_idx, _, _, _, _ = S.propose(net, n, frac, k, rank="random")
    r_trained, r_random = prop.recall(p_idx, truth), prop.recall(r_idx, truth)
    # (an offline fit of the same network shape to these features and
    # targets finds 90% of the top 20 at this budget; random choice 10%)
    assert r_trained >= 0.5 and r_trained >= r_random + 0.3, (r_trained, r_random)
    # every delta the proposal reports is the sweep's own value (batch-invariant walks)
    sweep_delta = dict(zip(truth.tolist(), deltas.tolist()))
    for i, d in zip(p_idx.tolist(), p_d.tolist()):
        if i in sweep_delta:
            assert d == sweep_delta[i]
    # the best trajectories' limits against the exact rational walk. The
    # largest deltas of a floating-point sweep include walks whose result
    # has lost the subdominant solution (the float ratios stop moving, so
    # delta is huge, while the exact limit is elsewhere, by 1e-5 relative
    # here): telling those apart is the exact confirmation's job, so it must
    # give a finite verdict for each and confirm some
    v = S.confirm(truth[:5], detail=True)
    assert np.isfinite(v["rel_err"]).all(), v["rel_err"]
    assert v["verified"].sum() >= 2, (v["rel_err"], v["floor"])
