"""Learned trajectory proposal for a delta search (BASELINE cfg 5).

A delta search over a seeded candidate set (cmfw.mlp's generator:
directions with components uniform in lo..hi over the family's axes, start
at the zeta point) either walks every candidate (the plain exhaustive sweep,
which stays the judge) or:

1. walks a training set of candidates disjoint from the searched ones and
   regresses their outcome with the tensor-core MLP (target: log1p-compressed
   delta where the walk is valid and delta finite, VALID_NAN for valid walks
   without a delta, FLOOR for invalid walks; valid rows weighted up);
2. scores every searched candidate with the network;
3. walks only the top-scoring candidates and keeps the best deltas;
4. confirms the reported results against the exact rational walk.

All walks, scoring and selection run on the GPU through the C ABI; GPU time
is summed from CUDA events around each enqueued stage.
"""
import numpy as np

from . import api, exact
from . import mlp as cm
from .mlp import FAMILY_INDEX

FLOOR = -3.0  # target of invalid walks
VALID_NAN = -2.0  # target of valid walks whose delta is undefined


def delta_target(delta):
    """Regression target of a finite delta: sign-preserving log1p, so that
    the rare huge deltas (exactly rational limits) do not dominate."""
    d = np.asarray(delta, np.float64)
    return (np.sign(d) * np.log1p(np.abs(d))).astype(np.float32)


class GpuClock:
    """Sums CUDA-event time of the stages recorded between start() and stop()."""

    def __init__(self):
        self.ms = 0.0

    def __enter__(self):
        torch = api._torch()
        self.a = torch.cuda.Event(enable_timing=True)
        self.b = torch.cuda.Event(enable_timing=True)
        self.a.record()
        return self

    def __exit__(self, *exc):
        self.b.record()
        self.b.synchronize()
        self.ms += self.a.elapsed_time(self.b)
        return False


def _walk_range(desc, seed, first, n, naxes, lo, hi, start, N, h, variant, batch, clock):
    """Walk candidates first .. first+n-1; returns (indices, delta, limit) of
    the valid ones with a finite delta, and the number valid."""
    torch = api._torch()
    keep_i, keep_d, keep_l = [], [], []
    n_valid = 0
    for b in range(0, n, batch):
        m = min(batch, n - b)
        with clock:
            idx = torch.arange(first + b, first + b + m, dtype=torch.int64, device="cuda")
            recs = cm.candidate_records(seed, idx, naxes, lo, hi, start)
            out = api.out_buffer(m)
            api.launch_walk(variant, desc, recs, out, m, N, h)
        res = api.records_from_device(out, m)
        v = res["valid"] == 1
        n_valid += int(v.sum())
        ok = v & np.isfinite(res["delta"])
        keep_i.append(np.nonzero(ok)[0] + first + b)
        keep_d.append(res["delta"][ok])
        keep_l.append(res["limit"][ok])
    cat = (lambda xs, dt: np.concatenate(xs) if xs else np.zeros(0, dt))
    return cat(keep_i, np.int64), cat(keep_d, np.float64), cat(keep_l, np.float64), n_valid


def _walk_indices(desc, seed, idx_dev, naxes, lo, hi, start, N, h, variant, batch, clock):
    torch = api._torch()
    keep_i, keep_d = [], []
    n_valid = 0
    n = int(idx_dev.numel())
    for b in range(0, n, batch):
        sub = idx_dev[b:b + batch]
        m = int(sub.numel())
        with clock:
            recs = cm.candidate_records(seed, sub, naxes, lo, hi, start)
            out = api.out_buffer(m)
            api.launch_walk(variant, desc, recs, out, m, N, h)
        res = api.records_from_device(out, m)
        v = res["valid"] == 1
        n_valid += int(v.sum())
        ok = v & np.isfinite(res["delta"])
        keep_i.append(sub.cpu().numpy()[ok])
        keep_d.append(res["delta"][ok])
    cat = (lambda xs, dt: np.concatenate(xs) if xs else np.zeros(0, dt))
    return cat(keep_i, np.int64), cat(keep_d, np.float64), n_valid


def top_k(idx, delta, k):
    o = np.argsort(-delta, kind="stable")[:k]
    return idx[o], delta[o]


class DeltaSearch:
    """One delta-search problem: family (p, q) at the zeta point, z = 1,
    candidates = directions with components uniform in lo..hi."""

    def __init__(self, p=8, q=7, lo=0, hi=4, N=1000, h=50, variant="df64", seed=20261203, batch=1 << 22):
        self.p, self.q, self.lo, self.hi, self.N, self.h = p, q, lo, hi, N, h
        self.naxes = p + q
        self.variant = variant
        self.seed = seed
        self.batch = batch
        self.desc = api.make_desc(p, q, 1.0)
        self.start = [1.0] * p + [2.0] * q
        self.family = FAMILY_INDEX[(p, q)]

    # -- the judge ------------------------------------------------------------
    def sweep(self, n, k=100):
        """Walk candidates 0 .. n-1; returns (top-k indices, their deltas,
        number valid, GPU ms)."""
        clock = GpuClock()
        idx, d, _, n_valid = _walk_range(self.desc, self.seed, 0, n, self.naxes, self.lo, self.hi, self.start, self.N,
                                         self.h, self.variant, self.batch, clock)
        ti, td = top_k(idx, d, k)
        return ti, td, n_valid, clock.ms

    # -- training -------------------------------------------------------------
    def training_set(self, n, offset):
        """Walk candidates offset .. offset+n-1 (disjoint from the searched
        ones); returns device records, family ids, targets, weights and GPU ms."""
        torch = api._torch()
        clock = GpuClock()
        targets = np.full(n, FLOOR, np.float32)
        weights = np.ones(n, np.float32)
        for b in range(0, n, self.batch):
            m = min(self.batch, n - b)
            with clock:
                idx = torch.arange(offset + b, offset + b + m, dtype=torch.int64, device="cuda")
                recs = cm.candidate_records(self.seed, idx, self.naxes, self.lo, self.hi, self.start)
                out = api.out_buffer(m)
                api.launch_walk(self.variant, self.desc, recs, out, m, self.N, self.h)
            res = api.records_from_device(out, m)
            valid = res["valid"] == 1
            ok = valid & np.isfinite(res["delta"])
            t = targets[b:b + m]
            t[valid] = VALID_NAN
            t[ok] = delta_target(res["delta"][ok])
        # the rare valid rows carry as much total weight as the invalid ones
        inf = targets > FLOOR
        if inf.any():
            weights[inf] = max(1.0, float((~inf).sum()) / float(inf.sum()))
        idx = torch.arange(offset, offset + n, dtype=torch.int64, device="cuda")
        recs = cm.candidate_records(self.seed, idx, self.naxes, self.lo, self.hi, self.start)
        fam = torch.full((n,), self.family, dtype=torch.int32, device="cuda")
        return recs, fam, torch.from_numpy(targets).cuda(), torch.from_numpy(weights).cuda(), clock.ms

    def train(self, net, data, epochs=3, batch=8192, lr=1e-3, seed=0):
        """Adam epochs over the training set in shuffled mini-batches; returns GPU ms."""
        torch = api._torch()
        recs, fam, y, w = data
        n = recs.shape[0]
        g = torch.Generator(device="cpu").manual_seed(seed)
        clock = GpuClock()
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g).cuda()
            for b in range(0, n - batch + 1, batch):
                sel = perm[b:b + batch]
                ws = float(w[sel].sum().item())
                with clock:
                    net.train_step(recs[sel], fam[sel], y[sel], w[sel], batch, ws, lr)
        net.status()
        return clock.ms

    # -- the proposal ---------------------------------------------------------
    def propose(self, net, n, fraction, k=100):
        """Score candidates 0 .. n-1, walk the top `fraction`, return (top-k
        indices, deltas, number walked, number valid, GPU ms by stage)."""
        torch = api._torch()
        scores = torch.empty(n, dtype=torch.float32, device="cuda")
        c_score, c_select, c_walk = GpuClock(), GpuClock(), GpuClock()
        with c_score:
            net.score_candidates(self.seed, 0, n, self.naxes, self.lo, self.hi, self.family, scores)
        n_walk = max(1, int(round(fraction * n)))
        with c_select:
            sel = cm.select_top(scores, n_walk)
        idx, d, n_valid = _walk_indices(self.desc, self.seed, sel, self.naxes, self.lo, self.hi, self.start, self.N,
                                        self.h, self.variant, self.batch, c_walk)
        ti, td = top_k(idx, d, k)
        net.status()
        return ti, td, int(sel.numel()), n_valid, {"score": c_score.ms, "select": c_select.ms, "walk": c_walk.ms}

    def confirm(self, indices, limits=None, rtol=1e-10, detail=False):
        """Exact check of the reported trajectories' f64 limits (the walk
        repeated in f64 with its limit source, against the exact rational
        walk); returns the number verified, or with detail=True the
        exact.verify record (errors and rounding floors per trajectory)."""
        torch = api._torch()
        if len(indices) == 0:
            return 0
        idx = torch.from_numpy(np.asarray(indices, np.int64)).cuda()
        recs_dev = cm.candidate_records(self.seed, idx, self.naxes, self.lo, self.hi, self.start)
        recs = recs_dev.cpu().numpy().reshape(-1).view(api.IN_DTYPE).copy()
        out, src = api.walk("f64", self.desc, recs, self.N, self.h, with_limit_src=True)
        v = exact.verify(self.desc, recs, out, src, self.N, self.h, rtol=rtol)
        return v if detail else int(v["verified"].sum())


def recall(found, truth):
    """Fraction of the judge's indices that the proposal also reports."""
    t = set(int(x) for x in truth)
    return (len(t & set(int(x) for x in found)) / len(t)) if t else 1.0
