"""Learned trajectory proposal: host interface of the tensor-core MLP
(include/cmfw.h, cmfw_mlp_*), plus the seeded candidate generator and the
top-k selection used to walk only the most promising directions.

Features of a trajectory: its direction components dir[0..14] / 4 and a
one-hot of the CMF family (FAMILY_INDEX). The network regresses a walk
outcome (the proposal's target, see cmfw.proposal)."""
import ctypes

import numpy as np

from . import api
from ._lib import MLP_SHAPES, OUT_DTYPE, check, lib

FAMILY_INDEX = {(3, 2): 0, (4, 3): 1, (5, 4): 2, (6, 5): 3, (8, 7): 4}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def unflatten(flat):
    out, off = [], 0
    for shp in MLP_SHAPES:
        n = int(np.prod(shp))
        out.append(np.asarray(flat[off:off + n], np.float32).reshape(shp))
        off += n
    return out


class Mlp:
    """A network on the current device with a batch capacity."""

    def __init__(self, max_batch=8192, seed=1):
        h = ctypes.c_void_p()
        check(lib().cmfw_mlp_create(int(max_batch), ctypes.c_uint64(seed), ctypes.byref(h)))
        self.h = h
        self.cap = (int(max_batch) + 127) // 128 * 128
        self.n_params = lib().cmfw_mlp_param_count()

    def close(self):
        if self.h:
            lib().cmfw_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        buf = np.zeros(self.n_params, np.float32)
        check(lib().cmfw_mlp_get_params(self.h, buf.ctypes.data_as(ctypes.c_void_p)))
        return buf

    def set_params(self, flat):
        buf = np.ascontiguousarray(flat, np.float32)
        assert buf.size == self.n_params
        check(lib().cmfw_mlp_set_params(self.h, buf.ctypes.data_as(ctypes.c_void_p)))

    def forward(self, d_in, d_family, n, stream=None):
        torch = api._torch()
        out = torch.empty(max(n, 1), dtype=torch.float32, device="cuda")
        check(lib().cmfw_mlp_forward(self.h, _ptr(d_in), _ptr(d_family), int(n), _ptr(out),
                                     api._stream_handle(stream)))
        return out[:n]

    def gradients(self, d_in, d_family, d_target, d_weight, n, weight_sum):
        g = np.zeros(self.n_params, np.float32)
        loss = ctypes.c_float(0)
        check(lib().cmfw_mlp_gradients(self.h, _ptr(d_in), _ptr(d_family), _ptr(d_target), _ptr(d_weight), int(n),
                                       ctypes.c_float(weight_sum), g.ctypes.data_as(ctypes.c_void_p),
                                       ctypes.byref(loss), api._stream_handle(None)))
        return g, loss.value

    def train_step(self, d_in, d_family, d_target, d_weight, n, weight_sum, lr, d_loss=None, stream=None):
        check(lib().cmfw_mlp_train_step(self.h, _ptr(d_in), _ptr(d_family), _ptr(d_target), _ptr(d_weight),
                                        int(n), ctypes.c_float(weight_sum), ctypes.c_float(lr), _ptr(d_loss),
                                        api._stream_handle(stream)))

    def train_epoch(self, d_in, d_family, d_target, d_weight, d_perm, batch, lr, d_loss=None, stream=None):
        """Adam steps over rows d_perm (int64 device tensor) `batch` at a
        time, full batches only, with no host synchronisation."""
        check(lib().cmfw_mlp_train_epoch(self.h, _ptr(d_in), _ptr(d_family), _ptr(d_target), _ptr(d_weight),
                                         _ptr(d_perm), int(d_perm.numel()), int(batch), ctypes.c_float(lr),
                                         _ptr(d_loss), api._stream_handle(stream)))

    def status(self):
        check(lib().cmfw_mlp_status(self.h))

    def score_candidates(self, seed, first, n, naxes, lo, hi, family, d_scores=None, stream=None, fused=True):
        """Scores of candidates first .. first+n-1: one fused launch (default)
        or per-layer tensor-core GEMMs through the activation buffers."""
        torch = api._torch()
        if d_scores is None:
            d_scores = torch.empty(max(n, 1), dtype=torch.float32, device="cuda")
        fn = lib().cmfw_mlp_score_candidates_fused if fused else lib().cmfw_mlp_score_candidates
        check(fn(self.h, ctypes.c_uint64(seed), int(first), int(n), int(naxes), int(lo), int(hi), int(family),
                 _ptr(d_scores), api._stream_handle(stream)))
        return d_scores[:n]

    def score_indices(self, seed, d_idx, naxes, lo, hi, family, d_scores=None, stream=None):
        """Scores of the candidates d_idx (int64 device tensor), one fused launch."""
        torch = api._torch()
        n = int(d_idx.numel())
        if d_scores is None:
            d_scores = torch.empty(max(n, 1), dtype=torch.float32, device="cuda")
        check(lib().cmfw_mlp_score_indices(self.h, ctypes.c_uint64(seed), _ptr(d_idx), n, int(naxes), int(lo),
                                           int(hi), int(family), _ptr(d_scores), api._stream_handle(stream)))
        return d_scores[:n]


def filter_candidates(desc, seed, first, n, lo, hi, start, N, h, steps=1, cap=None, stream=None):
    """Indices (int64 device tensor, ascending) of candidates first ..
    first+n-1 that pass the chunked walk's singularity filter; the others
    are invalid walks."""
    torch = api._torch()
    cap = int(cap if cap is not None else max(1024, n // 256))
    d_idx = torch.empty(max(cap, 1), dtype=torch.int64, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = (ctypes.c_double * 16)(*(list(start) + [0.0] * (16 - len(start))))
    check(lib().cmfw_filter_candidates(ctypes.byref(desc), ctypes.c_uint64(seed), int(first), int(n), int(lo),
                                       int(hi), st, int(N), int(h), int(steps), _ptr(d_idx), cap, _ptr(d_cnt),
                                       api._stream_handle(stream)))
    count = int(d_cnt.item())
    if count > cap:
        return filter_candidates(desc, seed, first, n, lo, hi, start, N, h, steps, 2 * count, stream)
    return torch.sort(d_idx[:count])[0]


def candidate_records(seed, d_idx, naxes, lo, hi, start, stream=None):
    """Device records of candidates d_idx (int64 tensor) of the seeded generator."""
    torch = api._torch()
    n = int(d_idx.numel())
    d_start = torch.tensor(list(start) + [0.0] * (16 - len(start)), dtype=torch.float64, device="cuda")
    out = torch.empty((max(n, 1), 192), dtype=torch.uint8, device="cuda")
    check(lib().cmfw_candidate_records(ctypes.c_uint64(seed), _ptr(d_idx), n, int(naxes), int(lo), int(hi),
                                       _ptr(d_start), _ptr(out), api._stream_handle(stream)))
    return out[:n]


def select_top(d_scores, k, cap=None):
    """Indices (int64 tensor, unordered) of the k largest scores; equal
    scores are taken in index order, so exactly min(k, n) are returned."""
    torch = api._torch()
    n = int(d_scores.numel())
    cap = int(cap or (2 * k + 1024))
    idx = torch.empty(cap, dtype=torch.int64, device="cuda")
    cnt = ctypes.c_int(0)
    check(lib().cmfw_select_top(_ptr(d_scores), n, int(k), _ptr(idx), cap, ctypes.byref(cnt),
                                api._stream_handle(None)))
    return idx[:min(cnt.value, cap)]
