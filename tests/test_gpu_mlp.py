"""Learned proposal network on the tensor cores (marked gpu): forward pass
and gradients of the library's tcgen05 kernels against the CPU reference
(oracle/mlp_ref.py, same BF16 roundings), training progress, the seeded
candidate generator and the top-k selection."""
import numpy as np
import pytest

import cmfw
from cmfw import mlp as cm
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    recs = np.zeros(n, dtype=cmfw.IN_DTYPE)
    recs["dir"][:, :15] = rng.integers(0, 5, (n, 15))
    fam = rng.integers(0, 5, n).astype(np.int32)
    return recs, fam


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_and_gradients_match_reference(cuda):
    torch = cuda
    m = cm.Mlp(512, seed=3)
    params = mlp_ref.unflatten(m.get_params())
    n = 300  # not a multiple of 128: padded rows must not leak into results
    recs, fam = _batch(n, 1)
    d_in, d_fam = cmfw.to_device(recs), torch.from_numpy(fam).cuda()
    X = mlp_ref.features(recs["dir"], fam)
    s_ref, _ = mlp_ref.forward(params, X)
    s = m.forward(d_in, d_fam, n).cpu().numpy()
    # the reference repeats the device's BF16 roundings; what remains is the
    # FP32 accumulation order (measured: forward <= 1e-4, gradients <= 4e-4)
    assert _rel(s, s_ref) < 1e-3, _rel(s, s_ref)
    rng = np.random.default_rng(2)
    y = rng.normal(0, 1, n).astype(np.float32)
    w = rng.uniform(0.5, 2.0, n).astype(np.float32)
    g, loss = m.gradients(d_in, d_fam, torch.from_numpy(y).cuda(), torch.from_numpy(w).cuda(), n, float(w.sum()))
    loss_ref, g_ref = mlp_ref.gradients(params, X, y, w, float(w.sum()))
    assert abs(loss - loss_ref) <= 1e-4 * abs(loss_ref)
    for name, a, b in zip(["W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4"], mlp_ref.unflatten(g),
                          mlp_ref.unflatten(g_ref)):
        assert _rel(a, b) < 3e-3, (name, _rel(a, b))
    # every batch sum is formed in a fixed order: the same bits again
    g2, loss2 = m.gradients(d_in, d_fam, torch.from_numpy(y).cuda(), torch.from_numpy(w).cuda(), n, float(w.sum()))
    assert np.array_equal(g, g2) and loss == loss2
    m.status()


def test_training_reduces_loss(cuda):
    torch = cuda
    m = cm.Mlp(1024, seed=5)
    n = 1024
    recs, fam = _batch(8 * n, 7)
    # a target the features determine: counts of x components equal to 4
    # and of y components equal to 0, and the family
    d = recs["dir"][:, :15]
    p = np.array(mlp_ref.FAMILY_P)[fam]
    ax = np.arange(15)[None, :]
    n4x = ((d == 4) & (ax < p[:, None])).sum(1)
    n0y = ((d == 0) & (ax >= p[:, None]) & (ax < 2 * p[:, None] - 1)).sum(1)
    y = (0.3 * n4x - 0.2 * n0y + 0.1 * fam).astype(np.float32)
    d_in, d_fam, d_y = cmfw.to_device(recs), torch.from_numpy(fam).cuda(), torch.from_numpy(y).cuda()
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    first = None
    for it in range(400):
        lo = (it % 8) * n
        m.train_step(d_in[lo:lo + n], d_fam[lo:lo + n], d_y[lo:lo + n], None, n, float(n), 2e-3, loss)
        if it == 0:
            first = float(loss.item())
    _, last = m.gradients(d_in[:n], d_fam[:n], d_y[:n], None, n, float(n))
    assert last < 0.05 * first, (first, last)
    m.status()


def test_train_epoch_matches_train_steps(cuda):
    """One epoch on the device (index gathers, device weight sums, fused
    Adam) trains the same network, bit for bit, as the same mini-batches
    stepped one call at a time: every sum over a batch is formed in a fixed
    order, and the weights (halves) sum exactly in any order. The same
    epoch without the weights (what a gather that lost them would train)
    ends elsewhere."""
    torch = cuda
    n, batch, lr = 4 * 1024 + 300, 1024, 2e-3  # the last partial batch is skipped
    recs, fam = _batch(n, 21)
    rng = np.random.default_rng(22)
    y = rng.normal(0, 1, n).astype(np.float32)
    w = (rng.integers(1, 5, n) / 2).astype(np.float32)
    d_in, d_fam = cmfw.to_device(recs), torch.from_numpy(fam).cuda()
    d_y, d_w = torch.from_numpy(y).cuda(), torch.from_numpy(w).cuda()
    perm = torch.randperm(n, generator=torch.Generator().manual_seed(3)).cuda()
    a, b, u = cm.Mlp(batch, seed=8), cm.Mlp(batch, seed=8), cm.Mlp(batch, seed=8)
    for _ in range(2):
        a.train_epoch(d_in, d_fam, d_y, d_w, perm, batch, lr)
        u.train_epoch(d_in, d_fam, d_y, None, perm, batch, lr)
        for s in range(0, n - batch + 1, batch):
            sel = perm[s:s + batch]
            b.train_step(d_in[sel], d_fam[sel], d_y[sel], d_w[sel], batch, float(d_w[sel].sum().item()), lr)
    p0 = cm.Mlp(batch, seed=8).get_params()
    pa, pb, pu = a.get_params(), b.get_params(), u.get_params()
    assert not np.array_equal(pa, p0)
    assert np.array_equal(pa, pb)
    assert _rel(pu - p0, pb - p0) > 1e-2, _rel(pu - p0, pb - p0)
    # and a second model trained the same way ends on the same bits
    c = cm.Mlp(batch, seed=8)
    for _ in range(2):
        c.train_epoch(d_in, d_fam, d_y, d_w, perm, batch, lr)
    assert np.array_equal(c.get_params(), pa)
    for m in (a, b, u, c):
        m.status()


def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    return x ^ (x >> np.uint64(31))


def test_candidates_and_selection(cuda):
    torch = cuda
    seed, naxes, lo, hi = 12345, 15, 0, 4
    m = cm.Mlp(4096, seed=9)
    idx = torch.arange(0, 3000, dtype=torch.int64, device="cuda")
    recs = cm.candidate_records(seed, idx, naxes, lo, hi, [1.0] * 8 + [2.0] * 7)
    host = recs.cpu().numpy().reshape(-1).view(cmfw.IN_DTYPE)
    with np.errstate(over="ignore"):
        i = np.arange(3000, dtype=np.uint64)[:, None]
        a = np.arange(naxes, dtype=np.uint64)[None, :]
        draw = _splitmix64(np.uint64(seed) ^ ((i * np.uint64(4) + (a >> np.uint64(2))) * np.uint64(0xD1B54A32D192ED03)))
        comp = lo + ((draw >> (np.uint64(16) * (a & np.uint64(3)))) & np.uint64(0xFFFF)) % np.uint64(hi - lo + 1)
    assert (host["dir"][:, :naxes] == comp.astype(np.int32)).all()
    assert (host["start"][:, :15] == [1.0] * 8 + [2.0] * 7).all()
    fam = torch.full((3000,), 4, dtype=torch.int32, device="cuda")
    a = m.forward(recs, fam, 3000)
    b = m.score_candidates(seed, 0, 3000, naxes, lo, hi, 4, fused=False)
    assert torch.equal(a, b)  # same features, same kernels
    # top-k over a million scores against a full sort
    rng = np.random.default_rng(4)
    sc = rng.normal(0, 1, 1_000_003).astype(np.float32)
    top = cm.select_top(torch.from_numpy(sc).cuda(), 1000).cpu().numpy()
    assert sorted(top.tolist()) == sorted(np.argsort(-sc)[:1000].tolist())
    # many equal scores (features that coincide): exactly k, equal scores by lower index
    tied = rng.integers(0, 50, 200_001).astype(np.float32)
    order = np.lexsort((np.arange(tied.size), -tied))
    for k in (1, 999, 4000, 200_001, 300_000):
        top = cm.select_top(torch.from_numpy(tied).cuda(), k).cpu().numpy()
        assert sorted(top.tolist()) == sorted(order[:k].tolist()), k


def test_fused_scoring_matches_layered_gemms(cuda):
    """The one-launch scoring (weights resident in a two-CTA cluster,
    activations exchanged through distributed shared memory) gives the
    per-layer GEMM path's scores."""
    torch = cuda
    m = cm.Mlp(1 << 16, seed=11)
    n = 100_003  # a partial last tile
    a = m.score_candidates(4242, 17, n, 15, 0, 4, 4, fused=False).cpu().numpy()
    b = m.score_candidates(4242, 17, n, 15, 0, 4, 4, fused=True).cpu().numpy()
    assert np.isfinite(b).all()
    np.testing.assert_allclose(b, a, rtol=1e-4, atol=1e-4 * float(np.abs(a).max()))
    m.status()
