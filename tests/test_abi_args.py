"""Argument checks of the C ABI's walk entry points, without a GPU.

Every entry point validates its arguments on the host before any CUDA call
(as the reference's programs check argv before touching the device), so
these calls return their status here: CMFW_EINVAL with a message for bad
arguments, CMFW_OK for an empty batch. No buffer passed below is ever
dereferenced.
"""
import ctypes

import numpy as np
import pytest

import cmfw
from cmfw._lib import Launch, check


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


# The calls below hand placeholder pointers to entry points that must
# reject them on the host; with a device present nothing is left to chance.
# (A string condition: evaluated only for tests that run.)
pytestmark = pytest.mark.skipif("_gpu_present()", reason="host-side checks only, run where no GPU is present")

MAX_DEPTH = 1 << 26  # CMFW_MAX_DEPTH
FAKE = ctypes.c_void_p(0x1000)  # a non-NULL pointer the checks must reject before use


def _status(rc):
    return cmfw._lib.STATUS_NAMES[rc]


def _walk(variant, desc, d_in, d_out, n, N=100, h=10, n_primes=8, launch=None):
    L = cmfw.lib()
    if variant == "rns":
        return L.cmfw_walk_rns(ctypes.byref(desc), d_in, d_out, n, N, h, n_primes,
                               ctypes.byref(launch) if launch else None, None)
    fn = L.cmfw_walk_f64 if variant == "f64" else L.cmfw_walk_df64
    return fn(ctypes.byref(desc), d_in, d_out, n, N, h, ctypes.byref(launch) if launch else None, None)


@pytest.mark.parametrize("variant", ["f64", "df64", "rns"])
def test_empty_batch_is_a_no_op(variant):
    assert _status(_walk(variant, cmfw.make_desc(3, 2, 0.5), None, None, 0)) == "OK"


@pytest.mark.parametrize("variant", ["f64", "df64", "rns"])
def test_bad_walk_arguments(variant):
    desc = cmfw.make_desc(3, 2, 0.5)
    L = cmfw.lib()
    assert _status(_walk(variant, desc, FAKE, FAKE, -1)) == "EINVAL"
    assert b"negative" in L.cmfw_last_error()
    assert _status(_walk(variant, desc, None, FAKE, 4)) == "EINVAL"
    assert b"NULL trajectory buffer" in L.cmfw_last_error()
    assert _status(_walk(variant, desc, FAKE, None, 4)) == "EINVAL"
    assert _status(_walk(variant, desc, FAKE, FAKE, 4, N=MAX_DEPTH + 1)) == "EINVAL"
    assert b"CMFW_MAX_DEPTH" in L.cmfw_last_error()
    bad = cmfw.make_desc(3, 2, 0.5)
    bad.rank = 9
    assert _status(_walk(variant, bad, FAKE, FAKE, 4)) == "EINVAL"


@pytest.mark.parametrize("variant", ["f64", "df64"])
def test_caller_workspace_too_small(variant):
    desc = cmfw.make_desc(6, 5, 1.0)
    need = cmfw.lib().cmfw_walk_workspace_bytes(ctypes.byref(desc), 100)
    assert need > 0
    launch = Launch()
    launch.d_workspace = FAKE.value
    launch.workspace_bytes = need - 1
    assert _status(_walk(variant, desc, FAKE, FAKE, 100, launch=launch)) == "EINVAL"
    assert b"below" in cmfw.lib().cmfw_last_error()


def test_workspace_bytes_grow_with_the_batch():
    L = cmfw.lib()
    d = cmfw.make_desc(6, 5, 1.0)
    a, b = L.cmfw_walk_workspace_bytes(ctypes.byref(d), 100), L.cmfw_walk_workspace_bytes(ctypes.byref(d), 200)
    assert 0 < a < b
    assert L.cmfw_walk_workspace_bytes(ctypes.byref(d), -1) == 0


@pytest.mark.parametrize("k", [0, 65])
def test_rns_modulus_count_checked_first(k):
    desc = cmfw.make_desc(3, 2, 0.5)
    assert _status(_walk("rns", desc, FAKE, FAKE, 4, n_primes=k)) == "EINVAL"
    assert b"n_primes" in cmfw.lib().cmfw_last_error()
    L = cmfw.lib()
    assert _status(L.cmfw_rns_trace(ctypes.byref(desc), FAKE, 4, 100, 10, k, 1, 0, FAKE, FAKE, None)) == "EINVAL"


def test_rns_trace_arguments():
    desc = cmfw.make_desc(3, 2, 0.5)
    L = cmfw.lib()
    assert _status(L.cmfw_rns_trace(ctypes.byref(desc), FAKE, 4, 100, 10, 8, 0, 0, FAKE, FAKE, None)) == "EINVAL"
    assert _status(L.cmfw_rns_trace(ctypes.byref(desc), FAKE, -1, 100, 10, 8, 1, 0, FAKE, FAKE, None)) == "EINVAL"
    assert _status(L.cmfw_rns_trace(ctypes.byref(desc), None, 0, 100, 10, 8, 1, 0, None, None, None)) == "OK"
    assert _status(L.cmfw_rns_trace(ctypes.byref(desc), FAKE, 4, 100, 10, 8, 1, 0, None, FAKE, None)) == "EINVAL"


def test_exact_walk_arguments():
    L = cmfw.lib()
    desc = cmfw.make_desc(3, 2, 0.5)
    args = lambda d, n, K: L.cmfw_exact_residues(ctypes.byref(d), FAKE, n, 100, 10, FAKE, K, None, FAKE, FAKE, None)
    assert _status(args(desc, 4, 0)) == "EINVAL"
    assert _status(args(desc, 4, 4097)) == "EINVAL"
    assert _status(args(desc, -1, 8)) == "EINVAL"
    assert _status(L.cmfw_exact_residues(ctypes.byref(desc), None, 0, 100, 10, None, 8, None, None, None,
                                         None)) == "OK"
    # the exact walk takes z = n / 2^k with |n| < 2^62 and k <= 62
    tiny = cmfw.make_desc(3, 2, 2.0 ** -70)
    assert _status(args(tiny, 4, 8)) == "EINVAL"
    assert b"dyadic" in L.cmfw_last_error()
    huge = cmfw.make_desc(3, 2, 2.0 ** 70)
    assert _status(args(huge, 4, 8)) == "EINVAL"


def test_host_entry_point_arguments():
    L = cmfw.lib()
    desc = cmfw.make_desc(3, 2, 0.5)
    recs = np.zeros(4, dtype=cmfw.IN_DTYPE)
    out = np.zeros(4, dtype=cmfw.OUT_DTYPE)
    kms, tms = ctypes.c_float(-1), ctypes.c_float(-1)
    call = lambda variant, n, k: L.cmfw_walk_host(cmfw._lib.VARIANTS[variant], ctypes.byref(desc),
                                                  recs.ctypes.data_as(ctypes.c_void_p),
                                                  out.ctypes.data_as(ctypes.c_void_p), n, 100, 10, k, None,
                                                  ctypes.byref(kms), ctypes.byref(tms))
    assert _status(call("rns", 4, 0)) == "EINVAL"
    assert _status(call("f64", -1, 8)) == "EINVAL"
    assert _status(call("f64", 0, 8)) == "OK"
    assert kms.value == 0.0 and tms.value == 0.0
    with pytest.raises(cmfw.CmfwError, match="EINVAL"):
        check(call("df64", -3, 8))


def test_reference_input_builder_arguments():
    L = cmfw.lib()
    buf = np.zeros(2, dtype=cmfw.IN_DTYPE)
    ptr = buf.ctypes.data_as(ctypes.c_void_p)
    assert _status(L.cmfw_reference_inputs(0, 2, 2, 0, 0, ptr)) == "EINVAL"
    assert _status(L.cmfw_reference_inputs(9, 8, 2, 0, 0, ptr)) == "EINVAL"
    assert _status(L.cmfw_reference_inputs(3, 2, -1, 0, 0, ptr)) == "EINVAL"
    assert _status(L.cmfw_reference_inputs(3, 2, 2, 0, 0, None)) == "EINVAL"
    assert _status(L.cmfw_reference_inputs(3, 2, 2, 1, 1, ptr)) == "OK"
