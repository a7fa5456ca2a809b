"""cmfw_walk_f64_noalloc: the f64 walk for callers that cannot call
cudaMalloc (all their device memory comes from another allocator's pool, or
they must not let a first allocation synchronise the device). Its scratch is
a fixed array in the library's device image instead of library-allocated
memory, so it must give the same results as cmfw_walk_f64 -- on two calls in
a row, the second of which reuses the array the first one left behind.

This file is collected last on purpose, and passes both alone in a fresh
process and after every other test."""
import ctypes

import numpy as np
import pytest

import cmfw
import cmfw.workloads as wl
from cmfw._lib import NOALLOC_SCRATCH_BYTES, CmfwError, check

pytestmark = pytest.mark.gpu


def _noalloc(desc, records, N, h):
    import torch
    n = len(records)
    d_in = cmfw.to_device(records)
    d_out = cmfw.out_buffer(n)
    d_out.fill_(0xA5)  # the entry point must write every output record
    st = cmfw.lib().cmfw_walk_f64_noalloc(ctypes.byref(desc), ctypes.c_void_p(d_in.data_ptr()),
                                         ctypes.c_void_p(d_out.data_ptr()), n, N, h,
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    check(st)
    torch.cuda.synchronize()
    return cmfw.records_from_device(d_out, n)


def _same(got, ref):
    np.testing.assert_array_equal(got["valid"], ref["valid"])
    np.testing.assert_array_equal(got["n_limits"], ref["n_limits"])
    m = ref["valid"] == 1
    for k in ("limit", "p", "q", "log_scale", "delta", "precision"):
        np.testing.assert_allclose(got[k][m], ref[k][m], rtol=1e-12, atol=0, equal_nan=True, err_msg=k)


def test_noalloc_matches_walk_f64_on_two_calls(cuda):
    # call 1: 6F5 zeta direction search; call 2: a smaller 3F2 batch, so any
    # state the first call left in the shared array would show
    d1 = cmfw.make_desc(6, 5, 1.0)
    r1 = wl.zeta_directions(6, 5, 3000, 11)
    d2 = cmfw.make_desc(3, 2, 0.5)
    r2 = wl.limit_starts(3, 2, 1500, 12)
    assert cmfw.lib().cmfw_walk_workspace_bytes(ctypes.byref(d1), len(r1)) <= NOALLOC_SCRATCH_BYTES
    got1 = _noalloc(d1, r1, 1000, 50)
    got2 = _noalloc(d2, r2, 1000, 50)
    _same(got1, cmfw.walk("f64", d1, r1, 1000, 50))
    _same(got2, cmfw.walk("f64", d2, r2, 1000, 50))
    assert (got1["valid"] == 1).sum() > 0 and (got2["valid"] == 1).sum() > 0


def test_noalloc_rejects_batches_beyond_the_fixed_array(cuda):
    desc = cmfw.make_desc(8, 7, 1.0)
    n = 100000
    assert cmfw.lib().cmfw_walk_workspace_bytes(ctypes.byref(desc), n) > NOALLOC_SCRATCH_BYTES
    recs = wl.zeta_directions(8, 7, 4, 3)
    d_in = cmfw.to_device(recs)
    d_out = cmfw.out_buffer(4)
    # sizes are checked before any device access, so n beyond the buffers is safe here
    st = cmfw.lib().cmfw_walk_f64_noalloc(ctypes.byref(desc), ctypes.c_void_p(d_in.data_ptr()),
                                         ctypes.c_void_p(d_out.data_ptr()), n, 1000, 50, None)
    with pytest.raises(CmfwError, match="fixed scratch"):
        check(st)
