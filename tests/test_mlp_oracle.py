"""The CPU reference of the proposal network (oracle/mlp_ref.py) against
finite differences in float64, and its BF16 rounding."""
import numpy as np

from oracle import mlp_ref as M


def test_reference_gradients_by_finite_differences():
    rng = np.random.default_rng(0)
    params = [rng.normal(0, 0.2, s) for s in M.SHAPES]
    X = rng.normal(0, 1, (9, 64))
    y = rng.normal(0, 1, 9)
    w = rng.uniform(0.5, 2, 9)
    _, g = M.gradients(params, X, y, w, bf16=False)
    flat = M.flatten(params)
    eps = 1e-6
    for i in rng.choice(len(flat), 60, replace=False):
        up, dn = flat.copy(), flat.copy()
        up[i] += eps
        dn[i] -= eps
        fd = (M.gradients(M.unflatten(up), X, y, w, bf16=False)[0]
              - M.gradients(M.unflatten(dn), X, y, w, bf16=False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005, -3.14159, 1e-40, np.inf], np.float32)
    r = M.to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0078125) and r[3] == np.float32(-3.140625)
    assert np.isinf(r[5])
    assert (r.view(np.uint32) & 0xFFFF == 0).all()
