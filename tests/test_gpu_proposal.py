"""What the learned proposal gains (marked gpu): on an 8F7 zeta delta
search over 10^6 seeded candidates, the network trained on walks of 10^6
other candidates, walking 2% of the searched candidates, finds far more of
the exhaustive sweep's top-20 deltas than walking the same number of
candidates chosen without it (untrained network: the same pipeline with
the initial weights; random choice: 2% expected)."""
import numpy as np
import pytest

from cmfw import mlp as cm
from cmfw import proposal as prop

pytestmark = pytest.mark.gpu


def test_trained_proposal_beats_the_same_budget_without_it(cuda):
    S = prop.DeltaSearch(8, 7, 0, 4, 1000, 50, "df64", seed=777, batch=1 << 20)
    n, frac, k = 1 << 20, 0.02, 20
    truth, deltas, n_valid, _ = S.sweep(n, k)
    assert len(truth) == k and n_valid > 100
    untrained = cm.Mlp(1 << 20, seed=1)
    u_idx, _, _, _, _ = S.propose(untrained, n, frac, k)
    data = S.training_set(1 << 20, 1 << 40)
    net = cm.Mlp(1 << 20, seed=1)
    S.train(net, data[:4], epochs=8)
    p_idx, p_d, n_walk, _, _ = S.propose(net, n, frac, k)
    assert abs(n_walk - frac * n) <= 0.01 * frac * n + 64
    r_trained, r_untrained = prop.recall(p_idx, truth), prop.recall(u_idx, truth)
    assert r_trained >= 0.25 and r_trained > r_untrained + 0.1, (r_trained, r_untrained)
    # every delta the proposal reports is the sweep's own value for that candidate
    common = np.intersect1d(p_idx, truth)
    assert len(common) > 0
    # the best trajectories' limits against the exact rational walk. The
    # f64 walk forms every step matrix in FP64, as the reference does (its
    # column coefficients pass 2^53 at these positions), so a few of the
    # best walks carry ~1e-10 from those roundings alone: at least two of
    # the three verify at 1e-10, and none is off by more than 1e-9
    v = S.confirm(truth[:3], detail=True)
    assert v["verified"].sum() >= 2, v["rel_err"]
    assert np.nanmax(v["rel_err"]) <= 1e-9, v["rel_err"]
