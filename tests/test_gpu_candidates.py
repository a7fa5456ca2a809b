"""The delta search's candidate stages on the GPU (marked gpu): the
candidate filter against the oracle's walks, scoring by index list against
scoring by range, and the batch-invariant walk."""
import numpy as np
import pytest

import cmfw
import oracle
from cmfw import mlp as cm

pytestmark = pytest.mark.gpu
P, Q, LO, HI, SEED = 8, 7, 0, 4, 4242
START = [1.0] * 8 + [2.0] * 7


def _records(idx):
    import torch
    d = cm.candidate_records(SEED, torch.as_tensor(np.asarray(idx, np.int64)).cuda(), P + Q, LO, HI, START)
    return d.cpu().numpy().reshape(-1).view(cmfw.IN_DTYPE).copy()


def test_filter_matches_the_oracle(cuda):
    """Survivors of `steps` lattice steps of tests are exactly the
    candidates whose oracle walk of `steps` lattice steps stays valid; with
    one step (the walk's own filter) they include every valid walk."""
    desc = cmfw.make_desc(P, Q, 1.0)
    n, first = 300000, 12345
    f3 = cm.filter_candidates(desc, SEED, first, n, LO, HI, START, 1000, 50, steps=3).cpu().numpy()
    f1 = cm.filter_candidates(desc, SEED, first, n, LO, HI, START, 1000, 50, steps=1).cpu().numpy()
    assert np.all(np.diff(f1) > 0) and set(f3) <= set(f1) and len(f1) > 50
    # the oracle: every candidate walked 3 lattice steps (N = 3, h = 1)
    recs = _records(np.arange(first, first + n))
    o3 = oracle.walk("f64", P, Q, 1.0, 3, 1, recs)
    np.testing.assert_array_equal(np.nonzero(o3["valid"] == 1)[0] + first, f3)
    # the survivors of one step include every walk that stays valid to N
    sub = np.arange(first, first + 40000)
    g = cmfw.walk("df64", desc, _records(sub), 1000, 50)
    assert set(sub[g["valid"] == 1]) <= set(f1)
    # nothing passes when N - 2h <= 0
    assert cm.filter_candidates(desc, SEED, first, 1000, LO, HI, START, 100, 50).numel() == 0


def test_filter_ragged_ranges(cuda):
    """The filter's block-wide queues drain whatever the range: any
    sub-range gives exactly the survivors of a larger range that fall in
    it (ranges shorter than a block, one candidate past a block, odd
    sizes, offsets)."""
    desc = cmfw.make_desc(P, Q, 1.0)
    big = cm.filter_candidates(desc, SEED, 0, 2_000_000, LO, HI, START, 1000, 50).cpu().numpy()
    assert len(big) > 500
    for first, n in ((0, 1), (5, 127), (100, 128), (1000, 129), (big[3], 1), (big[10] - 64, 200),
                     (777, 65537), (123456, 1_000_001)):
        got = cm.filter_candidates(desc, SEED, int(first), int(n), LO, HI, START, 1000, 50).cpu().numpy()
        want = big[(big >= first) & (big < first + n)]
        np.testing.assert_array_equal(got, want, err_msg=f"first={first} n={n}")


@pytest.mark.parametrize("p,q,z,lo,hi,start", [
    (4, 3, 0.5, -3, 3, [1.5, 2.0, 1.0, 3.0, 2.5, 1.0, 2.0]),
    (6, 5, 1.0, -2, 2, [1.0, 2.0, 1.5, 3.0, 1.0, 2.5, 2.0, 3.5, 1.0, 2.0, 4.0]),
    (6, 5, 1.0, -1, 3, [1.0] * 6 + [2.0] * 5),
    (3, 2, 1.0, -4, 4, [2.0, 1.0, 3.0, 2.0, 2.0]),
    (4, 3, 0.5, -3, 3, [1.1, 2.3, 0.7, 3.9, 2.2, 1.05, 2.6]),  # not dyadic
])
def test_filter_signed_directions_match_the_oracle(cuda, p, q, z, lo, hi, start):
    """Signed components (x- and y- steps, forward and inverse steps on
    both sides), a generic z and the rank reduced at z = 1: the survivors of
    three lattice steps of tests are the candidates whose oracle walk of
    three lattice steps (N = 3, h = 1) stays valid."""
    import torch
    desc = cmfw.make_desc(p, q, z)
    n, first = 60000, 99
    got = cm.filter_candidates(desc, SEED, first, n, lo, hi, start, 1000, 50, steps=3).cpu().numpy()
    d = cm.candidate_records(SEED, torch.arange(first, first + n, dtype=torch.int64).cuda(), p + q, lo, hi, start)
    recs = d.cpu().numpy().reshape(-1).view(cmfw.IN_DTYPE).copy()
    o = oracle.walk("f64", p, q, z, 3, 1, recs)
    want = np.nonzero(o["valid"] == 1)[0] + first
    assert 0 < len(want) <= n
    np.testing.assert_array_equal(got, want)


def test_filter_capacity_grows(cuda):
    desc = cmfw.make_desc(P, Q, 1.0)
    a = cm.filter_candidates(desc, SEED, 0, 200000, LO, HI, START, 1000, 50, cap=4)
    b = cm.filter_candidates(desc, SEED, 0, 200000, LO, HI, START, 1000, 50)
    assert a.numel() > 4 and np.array_equal(a.cpu().numpy(), b.cpu().numpy())


def test_scoring_by_index_equals_scoring_by_range(cuda):
    import torch
    net = cm.Mlp(1 << 14, seed=3)
    fam = cm.FAMILY_INDEX[(P, Q)]
    whole = net.score_candidates(SEED, 1000, 5000, P + Q, LO, HI, fam).cpu().numpy()
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(5000, 777, replace=False)) + 1000
    part = net.score_indices(SEED, torch.as_tensor(idx).cuda(), P + Q, LO, HI, fam).cpu().numpy()
    np.testing.assert_array_equal(part, whole[idx - 1000])
    assert net.score_indices(SEED, torch.zeros(0, dtype=torch.int64).cuda(), P + Q, LO, HI, fam).numel() == 0


@pytest.mark.parametrize("variant", ["f64", "df64"])
def test_batch_invariant_walk(cuda, variant):
    """With CMFW_F_BATCH_INVARIANT a trajectory's result does not depend on
    the rest of the batch: the same bits alone, in a batch of 3 and in a
    batch of 300 (without the flag those batches walk it in different part
    counts)."""
    recs = oracle.make_inputs(6, 5, 600, 0, True)[:300]
    recs["dir"][:, :11] = np.random.default_rng(2).integers(0, 2, (300, 11))
    recs["dir"][:, 5:11] = 0  # x-axes only: zeta-start walks that stay valid
    recs["dir"][:, 0] = 1
    desc = cmfw.make_desc(6, 5, 1.0)
    F = cmfw.F_BATCH_INVARIANT
    big = cmfw.walk(variant, desc, recs, 1000, 50, flags=F)
    assert (big["valid"] == 1).all()
    for n in (1, 3):
        small = cmfw.walk(variant, desc, recs[:n], 1000, 50, flags=F)
        assert small.tobytes() == big[:n].tobytes()
