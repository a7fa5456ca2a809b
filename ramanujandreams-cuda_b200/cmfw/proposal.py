"""Learned trajectory proposal for a delta search (BASELINE cfg 5).

A delta search over a seeded candidate set (cmfw.mlp's generator:
directions with components uniform in lo..hi over the family's axes, start
at the zeta point) starts with the walk's own singularity filter
(cmfw_filter_candidates: the position-only tests of the first lattice step,
drawn in place, no records): every candidate that fails it is an invalid
walk, and at a zeta start that is almost all of them. Then either

* the plain exhaustive sweep (the judge) walks every survivor, or
* the proposal scores the survivors with the tensor-core MLP and walks only
  the top `fraction` of them, keeping the best deltas.

The network is trained beforehand on walks of the survivors of a disjoint
candidate range. Its target is whether a survivor's delta is among the top
TOP_Q of the training walks' finite deltas (1 or 0, the rare positives
weighted to balance the rest), so that its output ranks survivors by how
likely they are to hold one of the search's best deltas; its features
(direction_features in csrc/candidates.cuh) count the x and y components
by magnitude, which the walk at the symmetric zeta start depends on.
Regressing the delta itself ranked the top no better than chance: deltas
span five orders of magnitude and the bulk of the loss is elsewhere.
Reported results are confirmed against the exact rational walk.

Every walk is batch-invariant (CMFW_F_BATCH_INVARIANT): a candidate's
delta is the same bits whether the sweep or the proposal walks it, so the
proposal's finds are the sweep's own values. All filtering, walks, scoring
and selection run on the GPU through the C ABI; GPU time is summed from
CUDA events around each enqueued stage, per stage.
"""
import numpy as np

from . import api, exact
from . import mlp as cm
from ._lib import F_BATCH_INVARIANT
from .mlp import FAMILY_INDEX

TOP_Q = 0.01  # training positives: the top 1% of the training walks' finite deltas


def top_target(valid, delta, top_q=TOP_Q):
    """Training target and weights from walk outcomes: 1 where the walk is
    valid and its delta finite and at least the (1 - top_q) quantile of the
    finite deltas, else 0; positives weighted so that both classes carry
    the same total weight. Returns (targets, weights, threshold)."""
    valid = np.asarray(valid, bool)
    delta = np.asarray(delta, np.float64)
    fin = valid & np.isfinite(delta)
    thr = float(np.quantile(delta[fin], 1.0 - top_q)) if fin.any() else np.inf
    pos = fin & (delta >= thr)
    t = pos.astype(np.float32)
    w = np.ones(len(t), np.float32)
    if pos.any() and (~pos).any():
        w[pos] = float((~pos).sum()) / float(pos.sum())
    return t, w, thr


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


def _walk_indices(desc, seed, idx_dev, naxes, lo, hi, start, N, h, variant, batch, clock):
    """Walk candidates idx_dev (int64 device tensor); returns (indices,
    deltas, limits) of the valid ones with a finite delta, the number valid,
    and every walked candidate's validity and delta (host arrays)."""
    keep_i, keep_d, keep_l, all_v, all_d = [], [], [], [], []
    n_valid = 0
    n = int(idx_dev.numel())
    for b in range(0, n, batch):
        sub = idx_dev[b:b + batch]
        m = int(sub.numel())
        with clock:
            recs = cm.candidate_records(seed, sub, naxes, lo, hi, start)
            out = api.out_buffer(m)
            api.launch_walk(variant, desc, recs, out, m, N, h, flags=F_BATCH_INVARIANT)
        res = api.records_from_device(out, m)
        v = res["valid"] == 1
        n_valid += int(v.sum())
        ok = v & np.isfinite(res["delta"])
        host = sub.cpu().numpy()
        keep_i.append(host[ok])
        keep_d.append(res["delta"][ok])
        keep_l.append(res["limit"][ok])
        all_v.append(v)
        all_d.append(res["delta"])
    cat = (lambda xs, dt: np.concatenate(xs) if xs else np.zeros(0, dt))
    return (cat(keep_i, np.int64), cat(keep_d, np.float64), cat(keep_l, np.float64), n_valid,
            cat(all_v, bool), cat(all_d, np.float64))


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

    def survivors(self, first, n, clock=None):
        """Candidates first .. first+n-1 that pass the walk's singularity
        filter (int64 device tensor, ascending)."""
        clock = clock or GpuClock()
        with clock:
            out = cm.filter_candidates(self.desc, self.seed, first, n, self.lo, self.hi, self.start, self.N, self.h)
        return out

    # -- the judge ------------------------------------------------------------
    def sweep(self, n, k=100):
        """Filter candidates 0 .. n-1 and walk every survivor; returns
        (top-k indices, their deltas, number valid, GPU ms, stage record)."""
        c_filter, c_walk = GpuClock(), GpuClock()
        surv = self.survivors(0, n, c_filter)
        idx, d, _, n_valid, _, _ = _walk_indices(self.desc, self.seed, surv, self.naxes, self.lo, self.hi,
                                                 self.start, self.N, self.h, self.variant, self.batch, c_walk)
        ti, td = top_k(idx, d, k)
        return ti, td, n_valid, c_filter.ms + c_walk.ms, {"filter_ms": c_filter.ms, "walk_ms": c_walk.ms,
                                                          "survivors": int(surv.numel())}

    # -- training -------------------------------------------------------------
    def training_set(self, n, offset):
        """Walk the survivors of candidates offset .. offset+n-1 (disjoint
        from the searched ones); returns device records, family ids,
        targets, weights and GPU ms."""
        torch = api._torch()
        clock = GpuClock()
        surv = self.survivors(offset, n, clock)
        _, _, _, _, valid, delta = _walk_indices(self.desc, self.seed, surv, self.naxes, self.lo, self.hi,
                                                 self.start, self.N, self.h, self.variant, self.batch, clock)
        m = int(surv.numel())
        targets, weights, thr = top_target(valid, delta)
        self.train_stats = {"walked": m, "valid": int(valid.sum()),
                            "finite_delta": int((valid & np.isfinite(delta)).sum()),
                            "positives": int(targets.sum()), "threshold": thr}
        recs = cm.candidate_records(self.seed, surv, self.naxes, self.lo, self.hi, self.start)
        fam = torch.full((m,), self.family, dtype=torch.int32, device="cuda")
        return recs, fam, torch.from_numpy(targets).cuda(), torch.from_numpy(weights).cuda(), clock.ms

    def train(self, net, data, epochs=30, batch=2048, lr=1e-3, seed=0):
        """Adam epochs over the training set in shuffled mini-batches; returns GPU ms."""
        torch = api._torch()
        recs, fam, y, w = data
        n = recs.shape[0]
        batch = min(batch, max(128, n // 4 // 128 * 128))
        g = torch.Generator(device="cpu").manual_seed(seed)
        clock = GpuClock()
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g).cuda()
            with clock:
                net.train_epoch(recs, fam, y, w, perm, batch, lr)
        net.status()
        return clock.ms

    # -- the proposal ---------------------------------------------------------
    def propose(self, net, n, fraction, k=100, rank="network", rng_seed=0):
        """Filter candidates 0 .. n-1, score the survivors, walk the top
        `fraction` of them; returns (top-k indices, deltas, number walked,
        number valid, GPU ms by stage). rank="random" walks the same number
        of survivors chosen without the network (the method without it)."""
        torch = api._torch()
        c_filter, c_score, c_select, c_walk = GpuClock(), GpuClock(), GpuClock(), GpuClock()
        surv = self.survivors(0, n, c_filter)
        m = int(surv.numel())
        n_walk = min(m, max(1, int(round(fraction * m))))
        # the chosen survivors are walked in ascending index order, as the
        # sweep walks them, so equal deltas rank alike in both top-k lists
        if rank == "random":
            g = torch.Generator(device="cpu").manual_seed(rng_seed)
            sel = surv[torch.sort(torch.randperm(m, generator=g)[:n_walk])[0].cuda()]
        else:
            with c_score:
                scores = net.score_indices(self.seed, surv, self.naxes, self.lo, self.hi, self.family)
            with c_select:
                sel = surv[torch.sort(cm.select_top(scores, n_walk))[0]] if m else surv
        idx, d, _, n_valid, _, _ = _walk_indices(self.desc, self.seed, sel, self.naxes, self.lo, self.hi,
                                                 self.start, self.N, self.h, self.variant, self.batch, c_walk)
        ti, td = top_k(idx, d, k)
        net.status()
        return ti, td, int(sel.numel()), n_valid, {"filter": c_filter.ms, "score": c_score.ms,
                                                   "select": c_select.ms, "walk": c_walk.ms, "survivors": m}

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
