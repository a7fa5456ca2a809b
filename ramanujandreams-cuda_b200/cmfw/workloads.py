"""Seeded synthetic workloads with the shapes and value ranges of the
benchmark configurations (the reference's published benchmark inputs are
reproduced separately by cmfw.reference_inputs).

All draws come from std::mt19937_64 (cmfw.mt64) so C++ and Python callers
produce identical records; a draw of "uniform in lo..hi" is
lo + (next() % (hi - lo + 1)).
"""
import numpy as np

from . import api
from ._lib import IN_DTYPE


class _Stream:
    """Sequential draws from one std::mt19937_64(seed) stream."""

    def __init__(self, seed, chunk=1 << 16):
        self.seed, self.chunk = seed, chunk
        self.offset = 0  # draws consumed so far
        self.buf = np.zeros(0, dtype=np.uint64)
        self.pos = 0

    def take(self, n):
        out = []
        while n > 0:
            if self.pos >= len(self.buf):
                self.buf = api.mt64(self.seed, self.chunk, offset=self.offset)
                self.pos = 0
            k = min(n, len(self.buf) - self.pos)
            out.append(self.buf[self.pos:self.pos + k])
            self.pos += k
            self.offset += k
            n -= k
        return np.concatenate(out) if out else np.zeros(0, dtype=np.uint64)


def zeta_start(p, q):
    """(1, ..., 1; 2, ..., 2), cmf_pfq.cuh:73-79."""
    return [1.0] * p + [2.0] * q


def limit_starts(p, q, n, seed, lo=1, hi=10):
    """Starts with every coordinate uniform in lo..hi, direction all ones."""
    s = _Stream(seed)
    recs = np.zeros(n, dtype=IN_DTYPE)
    draws = s.take(n * (p + q)).reshape(n, p + q)
    recs["start"][:, :p + q] = lo + (draws % np.uint64(hi - lo + 1)).astype(np.float64)
    recs["dir"][:, :p + q] = 1
    return recs


def zeta_directions(p, q, n, seed, lo=0, hi=3, offset=0):
    """Zeta start; direction components uniform in lo..hi (+ offset),
    redrawn while all are zero."""
    s = _Stream(seed)
    recs = np.zeros(n, dtype=IN_DTYPE)
    naxes = p + q
    recs["start"][:, :naxes] = zeta_start(p, q)
    span = np.uint64(hi - lo + 1)
    for i in range(n):
        while True:
            d = lo + (s.take(naxes) % span).astype(np.int64) + offset
            if d.any():
                break
        recs["dir"][i, :naxes] = d
    return recs


def valid_directions(p, q, n, seed, z=1.0, N=1000, h=50, lo=0, hi=3, offset=0, batch=1 << 16,
                     max_draws=1 << 26):
    """Non-degenerate variant of a zeta direction search: directions drawn as
    in zeta_directions from one seeded stream, kept only when the f64 walk at
    (z, N, h) stays valid, until n are kept (seeded rejection sampling; the
    validity test is the GPU walk, which agrees with the reference's validity
    trajectory for trajectory)."""
    s = _Stream(seed)
    naxes = p + q
    span = np.uint64(hi - lo + 1)
    desc = api.make_desc(p, q, z)
    kept, drawn, have = [], 0, 0
    while have < n:
        if drawn >= max_draws:
            raise RuntimeError(f"only {have} valid directions in {drawn} draws")
        d = lo + (s.take(batch * naxes) % span).astype(np.int64).reshape(batch, naxes) + offset
        d = d[d.any(axis=1)]  # all-zero draws are skipped, as in zeta_directions
        drawn += batch
        recs = np.zeros(len(d), dtype=IN_DTYPE)
        recs["start"][:, :naxes] = zeta_start(p, q)
        recs["dir"][:, :naxes] = d
        out = api.walk("f64", desc, recs, N, h)
        good = recs[out["valid"] == 1]
        kept.append(good)
        have += len(good)
    return np.concatenate(kept)[:n]


def config(name, seed=20261203):
    """Records and walk parameters of a named benchmark configuration."""
    if name == "cfg1":   # 3F2 f64 limit, z = 1/2, starts U{1..10}, dir 1^5
        return dict(p=3, q=2, z=0.5, N=1000, h=50, records=limit_starts(3, 2, 10000, seed))
    if name == "cfg2":   # 6F5 zeta delta search, dirs U{0..3}^11 != 0
        return dict(p=6, q=5, z=1.0, N=1000, h=50, records=zeta_directions(6, 5, 10000, seed))
    if name == "cfg3":   # 8F7 zeta limit, dir 1^15 + U{0..2}^15
        return dict(p=8, q=7, z=1.0, N=1000, h=50,
                    records=zeta_directions(8, 7, 10000, seed, lo=0, hi=2, offset=1))
    if name == "cfg2v":  # cfg2 restricted to directions whose walk stays valid
        return dict(p=6, q=5, z=1.0, N=1000, h=50, records=valid_directions(6, 5, 2000, seed))
    raise ValueError(name)


MIXED_FAMILIES = [(3, 2), (4, 3), (5, 4), (6, 5), (8, 7)]
MIXED_Z = [0.5, 1.0]


def mixed_batch(n, seed, N_lo=200, N_hi=5000, lo=1, hi=10, dlo=0, dhi=3):
    """Mixed batch: CMF family uniform over 3F2, 4F3, 5F4, 6F5, 8F7 and z
    uniform over {1/2, 1} (descriptor index = 2 * family + z index), start
    coordinates uniform in lo..hi, direction components uniform in dlo..dhi
    (redrawn while all are zero), depth N log-uniform in [N_lo, N_hi].

    Returns (descs, records, items) for cmfw.MixedBatch / cmfw.walk_mixed.
    """
    from ._lib import MIXED_ITEM_DTYPE
    descs = [api.make_desc(p, q, z) for (p, q) in MIXED_FAMILIES for z in MIXED_Z]
    s = _Stream(seed)
    recs = np.zeros(n, dtype=IN_DTYPE)
    items = np.zeros(n, dtype=MIXED_ITEM_DTYPE)
    head = s.take(3 * n).reshape(n, 3)
    fam = (head[:, 0] % np.uint64(len(MIXED_FAMILIES))).astype(np.int64)
    zi = (head[:, 1] % np.uint64(len(MIXED_Z))).astype(np.int64)
    u = (head[:, 2] >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    items["desc"] = 2 * fam + zi
    items["N"] = np.floor(N_lo * (N_hi / N_lo) ** u).astype(np.int32)
    span = np.uint64(hi - lo + 1)
    dspan = np.uint64(dhi - dlo + 1)
    for i in range(n):
        p, q = MIXED_FAMILIES[fam[i]]
        na = p + q
        recs["start"][i, :na] = lo + (s.take(na) % span).astype(np.float64)
        while True:
            d = dlo + (s.take(na) % dspan).astype(np.int64)
            if d.any():
                break
        recs["dir"][i, :na] = d
    return descs, recs, items
