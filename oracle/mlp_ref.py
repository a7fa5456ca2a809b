"""CPU reference of the learned-proposal MLP -- TEST INFRASTRUCTURE.

numpy restatement of the network computed by the library's tensor-core
kernels (cmfw_mlp_*): features, forward, weighted squared-error loss and
backward, with the same BF16 roundings as the device path when `bf16=True`
(weights, activations H1..H3 and the pre-activation gradients are rounded
to BF16; products accumulate in FP32). With `bf16=False` and float64
inputs it is the exact mathematics, which tests check by finite
differences. Parameter order: W1 [256 x 64], b1, W2, b2, W3, b3, w4, b4.
"""
import numpy as np

SHAPES = [(256, 64), (256,), (256, 256), (256,), (256, 256), (256,), (256,), (1,)]


def to_bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


def unflatten(flat):
    out, off = [], 0
    for shp in SHAPES:
        n = int(np.prod(shp))
        out.append(np.asarray(flat[off:off + n]).reshape(shp))
        off += n
    return out


def flatten(parts):
    return np.concatenate([np.asarray(p).reshape(-1) for p in parts])


FAMILY_P = [3, 4, 5, 6, 8]


def features(dirs, family):
    """X [n x 64], as the device's direction_features (csrc/candidates.cuh):
    for the x components (the family's first p axes) and the y components
    (the next q = p - 1), how many have |d| = 0, 1, 2, 3 and >= 4, over p
    (columns 0..4) and over q (5..9); the negative ones over p and q (10,
    11); one-hot(family) at 15..19; zeros elsewhere; rounded to BF16."""
    dirs = np.asarray(dirs)
    family = np.asarray(family)
    n = len(dirs)
    X = np.zeros((n, 64), np.float32)
    for t in range(n):
        p = FAMILY_P[int(family[t])]
        q = p - 1
        d = dirs[t, :p + q].astype(np.int64)
        m = np.minimum(np.abs(d), 4)
        ip, iq = np.float32(1.0) / np.float32(p), np.float32(1.0) / np.float32(q)
        for k in range(5):
            X[t, k] = np.float32((m[:p] == k).sum()) * ip
            X[t, 5 + k] = np.float32((m[p:] == k).sum()) * iq
        X[t, 10] = np.float32((d[:p] < 0).sum()) * ip
        X[t, 11] = np.float32((d[p:] < 0).sum()) * iq
        X[t, 15 + int(family[t])] = 1.0
    return to_bf16(X)  # the device holds features in BF16


def forward(params, X, bf16=True):
    W1, b1, W2, b2, W3, b3, w4, b4 = params
    q = to_bf16 if bf16 else (lambda a: a)
    dt = np.float32 if bf16 else np.float64
    X = X.astype(dt)
    acts = [X]
    h = X
    for W, b in ((W1, b1), (W2, b2), (W3, b3)):
        z = h @ q(W.astype(dt)).T.astype(dt) + b.astype(dt)
        h = q(np.maximum(z, 0)).astype(dt)
        acts.append(h)
    score = h @ w4.astype(dt) + b4.astype(dt)[0]
    return score, acts


def gradients(params, X, y, w=None, wsum=None, bf16=True):
    """Loss and flattened gradients of sum w (s - y)^2 / wsum."""
    W1, b1, W2, b2, W3, b3, w4, b4 = params
    q = to_bf16 if bf16 else (lambda a: a)
    dt = np.float32 if bf16 else np.float64
    score, acts = forward(params, X, bf16)
    n = len(X)
    w = np.ones(n, dt) if w is None else np.asarray(w, dt)
    wsum = float(w.sum()) if wsum is None else float(wsum)
    r = score - np.asarray(y, dt)
    loss = float((w * r * r).sum() / wsum)
    ds = (2.0 * w * r / wsum).astype(dt)
    H1, H2, H3 = acts[1], acts[2], acts[3]
    gw4 = ds @ H3
    gb4 = np.array([ds.sum()], dt)
    dZ = q(np.outer(ds, w4.astype(dt)) * (H3 > 0)).astype(dt)
    grads = {}
    Ws = [W1, W2, W3]
    for l in (2, 1, 0):
        grads[2 * l + 1] = dZ.sum(0)
        grads[2 * l] = dZ.T @ acts[l]
        if l > 0:
            dZ = q((dZ @ q(Ws[l].astype(dt)).astype(dt)) * (acts[l] > 0)).astype(dt)
    grads[6], grads[7] = gw4, gb4
    return loss, flatten([grads[i] for i in range(8)])
