"""Loads libcmfw.so (the C ABI of include/cmfw.h) and declares its signatures.

The library is built in-tree by ``make -C ramanujandreams-cuda_b200``; there
is no fallback implementation: if the library is missing, every call raises.
"""
import ctypes
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libcmfw.so")
BIN_DIR = os.path.join(PKG_ROOT, "bin")

IN_DTYPE = np.dtype([("dir", "<i4", 16), ("start", "<f8", 16)])
OUT_DTYPE = np.dtype([("limit", "<f8"), ("delta", "<f8"), ("p", "<f8"), ("q", "<f8"),
                      ("precision", "<f8"), ("log_scale", "<f8"), ("valid", "<i4"),
                      ("n_limits", "<i4")])
MIXED_ITEM_DTYPE = np.dtype([("desc", "<i4"), ("N", "<i4")])
assert IN_DTYPE.itemsize == 192 and OUT_DTYPE.itemsize == 56
MAX_MIXED_DESCS = 16
MLP_IN, MLP_HIDDEN = 64, 256
# flattened parameter shapes: W1, b1, W2, b2, W3, b3, w4, b4
MLP_SHAPES = [(256, 64), (256,), (256, 256), (256,), (256, 256), (256,), (256,), (1,)]

CMFW_OK = 0
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ENOMEM", 4: "ETIMEOUT", 5: "EUNSUPPORTED"}
TRAJ_STATUS = {0: "ok", 1: "singular_lead", 2: "singular_denom", 3: "singular_solve",
               4: "nonfinite", 5: "bad_depth", 6: "step_cap", 7: "modulus_zero",
               8: "not_integral", 9: "bad_family"}

F_DF64_COMPAT = 0x1
F_UNFUSED_COLUMN = 0x2
F_SEQUENTIAL = 0x4
F_PLAIN_RUNS = 0x8
F_BATCH_INVARIANT = 0x10
NOALLOC_SCRATCH_BYTES = 32 << 20  # CMFW_NOALLOC_SCRATCH_BYTES

VARIANTS = {"f64": 0, "df64": 1, "rns": 2}

# Every symbol include/cmfw.h declares.
EXPORTS = [
    "cmfw_version", "cmfw_last_error", "cmfw_make_desc", "cmfw_check_desc",
    "cmfw_walk_workspace_bytes", "cmfw_walk_f64", "cmfw_walk_f64_noalloc", "cmfw_walk_df64", "cmfw_walk_rns",
    "cmfw_rns_trace", "cmfw_exact_residues", "cmfw_exact_recon_words", "cmfw_exact_reconstruct",
    "cmfw_reference_inputs", "cmfw_mt64_fill",
    "cmfw_mt64_fill_at", "cmfw_walk_host", "cmfw_pipe_peak", "cmfw_device_banner", "cmfw_device_meminfo",
    "cmfw_mixed_workspace_bytes", "cmfw_walk_mixed", "cmfw_mixed_autotune", "cmfw_mixed_graph_create",
    "cmfw_mixed_graph_launch", "cmfw_mixed_graph_destroy",
    "cmfw_mlp_create", "cmfw_mlp_destroy", "cmfw_mlp_param_count", "cmfw_mlp_get_params", "cmfw_mlp_set_params",
    "cmfw_mlp_forward", "cmfw_mlp_gradients", "cmfw_mlp_train_step", "cmfw_mlp_train_epoch", "cmfw_mlp_status",
    "cmfw_mlp_score_candidates", "cmfw_mlp_score_candidates_fused", "cmfw_mlp_score_indices",
    "cmfw_filter_candidates", "cmfw_candidate_records", "cmfw_select_top",
]


class CmfwError(RuntimeError):
    """A cmfw_* call returned a status other than CMFW_OK."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Desc(ctypes.Structure):
    """cmfw_desc (CMFDesc, cmf_pfq.cuh:41-47)."""
    _fields_ = [("p", ctypes.c_int), ("q", ctypes.c_int), ("rank", ctypes.c_int),
                ("naxes", ctypes.c_int), ("z", ctypes.c_double)]


class Launch(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int), ("flags", ctypes.c_int),
                ("d_status", ctypes.c_void_p), ("d_workspace", ctypes.c_void_p),
                ("workspace_bytes", ctypes.c_size_t), ("d_limit_src", ctypes.c_void_p),
                ("ev_main_start", ctypes.c_void_p), ("ev_main_stop", ctypes.c_void_p)]


class MixedTile(ctypes.Structure):
    """cmfw_mixed_tile: one descriptor's launch shape in a mixed batch."""
    _fields_ = [("block_size", ctypes.c_int), ("grab", ctypes.c_int), ("ctas_per_sm", ctypes.c_int)]


class MixedTuning(ctypes.Structure):
    """cmfw_mixed_tuning."""
    _fields_ = [("persistent", ctypes.c_int), ("tile", MixedTile * 16), ("prescan", ctypes.c_int)]


_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_ROOT}` "
                               "(the CMF walk has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        vp, ci, cd, cs = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
        P = ctypes.POINTER
        L.cmfw_version.restype = ctypes.c_char_p
        L.cmfw_last_error.restype = ctypes.c_char_p
        L.cmfw_make_desc.restype = Desc
        L.cmfw_make_desc.argtypes = [ci, ci, cd]
        L.cmfw_check_desc.argtypes = [P(Desc)]
        L.cmfw_walk_workspace_bytes.restype = cs
        L.cmfw_walk_workspace_bytes.argtypes = [P(Desc), ci]
        for name in ("cmfw_walk_f64", "cmfw_walk_df64"):
            getattr(L, name).argtypes = [P(Desc), vp, vp, ci, ci, ci, P(Launch), vp]
        L.cmfw_walk_f64_noalloc.argtypes = [P(Desc), vp, vp, ci, ci, ci, vp]
        L.cmfw_walk_rns.argtypes = [P(Desc), vp, vp, ci, ci, ci, ci, P(Launch), vp]
        L.cmfw_rns_trace.argtypes = [P(Desc), vp, ci, ci, ci, ci, ci, ci, vp, vp, vp]
        L.cmfw_exact_residues.argtypes = [P(Desc), vp, ci, ci, ci, vp, ci, vp, vp, vp, vp]
        L.cmfw_exact_recon_words.argtypes = [ci]
        L.cmfw_exact_reconstruct.argtypes = [vp, vp, vp, ci, ci, ci, vp, vp, vp, vp, vp, vp, vp]
        L.cmfw_reference_inputs.argtypes = [ci, ci, ci, ci, ci, vp]
        L.cmfw_mt64_fill.argtypes = [ctypes.c_uint64, vp, cs]
        L.cmfw_mt64_fill.restype = None
        L.cmfw_mt64_fill_at.argtypes = [ctypes.c_uint64, ctypes.c_uint64, vp, cs]
        L.cmfw_mt64_fill_at.restype = None
        L.cmfw_walk_host.argtypes = [ci, P(Desc), vp, vp, ci, ci, ci, ci, P(Launch),
                                     P(ctypes.c_float), P(ctypes.c_float)]
        L.cmfw_device_banner.argtypes = [ctypes.c_char_p, cs]
        L.cmfw_pipe_peak.argtypes = [ci, P(ctypes.c_double)]
        L.cmfw_device_meminfo.argtypes = [P(cs), P(cs)]
        L.cmfw_mixed_workspace_bytes.restype = cs
        L.cmfw_mixed_workspace_bytes.argtypes = [ci, ci]
        L.cmfw_walk_mixed.argtypes = [P(Desc), ci, vp, vp, vp, ci, ci, ci, P(MixedTuning), P(Launch), vp]
        L.cmfw_mixed_autotune.argtypes = [P(Desc), ci, vp, vp, vp, ci, ci, ci, P(Launch), ci, P(MixedTuning), vp]
        L.cmfw_mixed_graph_create.argtypes = [P(Desc), ci, vp, vp, vp, ci, ci, ci, P(MixedTuning), P(Launch),
                                              P(vp)]
        L.cmfw_mixed_graph_launch.argtypes = [vp, vp]
        L.cmfw_mixed_graph_destroy.argtypes = [vp]
        L.cmfw_mixed_graph_destroy.restype = None
        fp, ll, u64 = ctypes.c_float, ctypes.c_longlong, ctypes.c_uint64
        L.cmfw_mlp_create.argtypes = [ci, u64, P(vp)]
        L.cmfw_mlp_destroy.argtypes = [vp]
        L.cmfw_mlp_destroy.restype = None
        L.cmfw_mlp_param_count.restype = cs
        L.cmfw_mlp_get_params.argtypes = [vp, vp]
        L.cmfw_mlp_set_params.argtypes = [vp, vp]
        L.cmfw_mlp_forward.argtypes = [vp, vp, vp, ci, vp, vp]
        L.cmfw_mlp_gradients.argtypes = [vp, vp, vp, vp, vp, ci, fp, vp, vp, vp]
        L.cmfw_mlp_train_step.argtypes = [vp, vp, vp, vp, vp, ci, fp, fp, vp, vp]
        L.cmfw_mlp_train_epoch.argtypes = [vp, vp, vp, vp, vp, vp, ll, ci, fp, vp, vp]
        L.cmfw_mlp_status.argtypes = [vp]
        L.cmfw_mlp_score_candidates.argtypes = [vp, u64, ll, ll, ci, ci, ci, ci, vp, vp]
        L.cmfw_mlp_score_candidates_fused.argtypes = [vp, u64, ll, ll, ci, ci, ci, ci, vp, vp]
        L.cmfw_mlp_score_indices.argtypes = [vp, u64, vp, ll, ci, ci, ci, ci, vp, vp]
        L.cmfw_filter_candidates.argtypes = [P(Desc), u64, ll, ll, ci, ci, vp, ci, ci, ci, vp, ll, vp, vp]
        L.cmfw_candidate_records.argtypes = [u64, vp, ci, ci, ci, ci, vp, vp, vp]
        L.cmfw_select_top.argtypes = [vp, ll, ll, vp, ci, P(ci), vp]
        _lib = L
    return _lib


def check(status):
    if status != CMFW_OK:
        raise CmfwError(status, lib().cmfw_last_error().decode())
