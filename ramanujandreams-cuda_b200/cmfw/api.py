"""Python host interface over the C ABI.

Mirrors the reference's per-variant operation -- build trajectory records,
run one walk over them, read back one result record per trajectory
(cmf_walk_{f64,df64,rns}.cu run_benchmark) -- with the walk itself always on
the GPU through libcmfw.so. torch supplies device memory and streams only.
"""
import ctypes

import numpy as np

from ._lib import (IN_DTYPE, MIXED_ITEM_DTYPE, OUT_DTYPE, VARIANTS, Desc, Launch, MixedTuning, check, lib)


def make_desc(p, q, z):
    """cmfw_make_desc (make_cmf_desc, cmf_pfq.cuh:50-61)."""
    return lib().cmfw_make_desc(int(p), int(q), float(z))


def check_desc(desc):
    check(lib().cmfw_check_desc(ctypes.byref(desc)))


def version():
    return lib().cmfw_version().decode()


def reference_inputs(p, q, n, mode, use_zeta):
    """Input records exactly as the reference programs build them."""
    out = np.zeros(n, dtype=IN_DTYPE)
    check(lib().cmfw_reference_inputs(p, q, n, int(mode), int(bool(use_zeta)),
                                      out.ctypes.data_as(ctypes.c_void_p)))
    return out


def mt64(seed, n, offset=0):
    """Outputs offset .. offset+n-1 of std::mt19937_64(seed)."""
    out = np.zeros(n, dtype=np.uint64)
    lib().cmfw_mt64_fill_at(ctypes.c_uint64(seed), ctypes.c_uint64(offset),
                            out.ctypes.data_as(ctypes.c_void_p), n)
    return out


def _torch():
    import torch
    return torch


def _stream_handle(stream):
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def to_device(records):
    """Copy IN_DTYPE records (numpy) to a device uint8 tensor of n x 192 bytes."""
    torch = _torch()
    arr = np.ascontiguousarray(records, dtype=IN_DTYPE)
    return torch.from_numpy(arr.view(np.uint8).reshape(len(arr), IN_DTYPE.itemsize)).cuda()


def out_buffer(n):
    torch = _torch()
    return torch.empty((max(n, 1), OUT_DTYPE.itemsize), dtype=torch.uint8, device="cuda")


def records_from_device(buf, n):
    host = buf[:n].cpu().numpy()
    return host.reshape(-1).view(OUT_DTYPE).copy()


def launch_walk(variant, desc, d_in, d_out, n, N, h, n_primes=8, flags=0, block_size=0,
                d_status=None, d_limit_src=None, d_workspace=None, stream=None, main_events=None):
    """Enqueue one walk on device buffers (torch tensors); no synchronisation.
    main_events: an optional pair of recorded torch.cuda.Event (timing
    enabled) that the library records around the walk's main kernel."""
    L = lib()
    launch = Launch()
    launch.block_size = block_size
    launch.flags = flags
    if main_events is not None:
        launch.ev_main_start = main_events[0].cuda_event
        launch.ev_main_stop = main_events[1].cuda_event
    launch.d_status = d_status.data_ptr() if d_status is not None else None
    launch.d_limit_src = d_limit_src.data_ptr() if d_limit_src is not None else None
    if d_workspace is not None:
        launch.d_workspace = d_workspace.data_ptr()
        launch.workspace_bytes = d_workspace.numel() * d_workspace.element_size()
    s = _stream_handle(stream)
    pin, pout = ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr())
    if variant == "f64":
        st = L.cmfw_walk_f64(ctypes.byref(desc), pin, pout, n, N, h, ctypes.byref(launch), s)
    elif variant == "df64":
        st = L.cmfw_walk_df64(ctypes.byref(desc), pin, pout, n, N, h, ctypes.byref(launch), s)
    elif variant == "rns":
        st = L.cmfw_walk_rns(ctypes.byref(desc), pin, pout, n, N, h, n_primes, ctypes.byref(launch), s)
    else:
        raise ValueError(f"unknown variant {variant!r}")
    check(st)


def walk(variant, desc, records, N, h, n_primes=8, flags=0, block_size=0, with_status=False,
         with_limit_src=False):
    """Walk numpy records on the GPU and return numpy result records.

    Returns OUT_DTYPE records, plus the per-trajectory status codes and/or
    limit-source codes when requested.
    """
    torch = _torch()
    n = len(records)
    d_in = to_device(records) if n else torch.empty((1, 192), dtype=torch.uint8, device="cuda")
    d_out = out_buffer(n)
    d_status = torch.empty(max(n, 1), dtype=torch.uint8, device="cuda") if with_status else None
    d_src = torch.empty(max(n, 1), dtype=torch.int32, device="cuda") if with_limit_src else None
    launch_walk(variant, desc, d_in, d_out, n, N, h, n_primes, flags, block_size, d_status, d_src)
    torch.cuda.synchronize()
    res = [records_from_device(d_out, n)]
    if with_status:
        res.append(d_status[:n].cpu().numpy())
    if with_limit_src:
        res.append(d_src[:n].cpu().numpy())
    return res[0] if len(res) == 1 else tuple(res)


def walk_host(variant, desc, records, N, h, n_primes=8, flags=0, block_size=0):
    """cmfw_walk_host: host buffers in and out; returns (results, kernel_ms, total_ms)."""
    recs = np.ascontiguousarray(records, dtype=IN_DTYPE)
    n = len(recs)
    out = np.zeros(max(n, 1), dtype=OUT_DTYPE)
    launch = Launch()
    launch.block_size = block_size
    launch.flags = flags
    kms, tms = ctypes.c_float(0), ctypes.c_float(0)
    check(lib().cmfw_walk_host(VARIANTS[variant], ctypes.byref(desc),
                               recs.ctypes.data_as(ctypes.c_void_p),
                               out.ctypes.data_as(ctypes.c_void_p), n, N, h, n_primes,
                               ctypes.byref(launch), ctypes.byref(kms), ctypes.byref(tms)))
    return out[:n], kms.value, tms.value


def rns_trace(desc, records, N, h, n_primes, steps, flags=0):
    """Compat-RNS residue matrices after `steps` steps: (res[n, K, rank, rank], ok[n])."""
    torch = _torch()
    n = len(records)
    d_in = to_device(records)
    r = desc.rank
    d_res = torch.zeros((n, n_primes, r, r), dtype=torch.int32, device="cuda")
    d_ok = torch.zeros(n, dtype=torch.int32, device="cuda")
    check(lib().cmfw_rns_trace(ctypes.byref(desc), ctypes.c_void_p(d_in.data_ptr()), n, N, h,
                               n_primes, steps, flags, ctypes.c_void_p(d_res.data_ptr()),
                               ctypes.c_void_p(d_ok.data_ptr()), _stream_handle(None)))
    torch.cuda.synchronize()
    return d_res.cpu().numpy().view(np.uint32), d_ok.cpu().numpy().astype(bool)


def exact_residues(desc, records, N, h, primes, pairs=None, d_in=None):
    """Exact walk residues: (res[n, 3, 2, K] uint32, prime_ok[n, K] bool)."""
    torch = _torch()
    n = len(records) if d_in is None else d_in.shape[0]
    if d_in is None:
        d_in = to_device(records)
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    K = len(primes)
    d_primes = torch.from_numpy(primes.view(np.int32)).cuda()
    d_res = torch.zeros((n, 3, 2, K), dtype=torch.int32, device="cuda")
    d_ok = torch.zeros((n, K), dtype=torch.uint8, device="cuda")
    d_pairs = None
    if pairs is not None:
        d_pairs = torch.from_numpy(np.ascontiguousarray(pairs, dtype=np.int32)).cuda()
    check(lib().cmfw_exact_residues(
        ctypes.byref(desc), ctypes.c_void_p(d_in.data_ptr()), n, N, h,
        ctypes.c_void_p(d_primes.data_ptr()), K,
        ctypes.c_void_p(d_pairs.data_ptr()) if d_pairs is not None else None,
        ctypes.c_void_p(d_res.data_ptr()), ctypes.c_void_p(d_ok.data_ptr()), _stream_handle(None)))
    torch.cuda.synchronize()
    return d_res.cpu().numpy().view(np.uint32), d_ok.cpu().numpy().astype(bool)


def exact_residues_device(desc, d_in, n, N, h, primes, pairs=None):
    """cmfw_exact_residues into device tensors: (d_res [n, 3, 2, K] int32
    view of uint32, d_ok [n, K] uint8, d_primes)."""
    torch = _torch()
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    K = len(primes)
    d_primes = torch.from_numpy(primes.view(np.int32)).cuda()
    d_res = torch.zeros((max(n, 1), 3, 2, K), dtype=torch.int32, device="cuda")
    d_ok = torch.zeros((max(n, 1), K), dtype=torch.uint8, device="cuda")
    d_pairs = None
    if pairs is not None:
        d_pairs = torch.from_numpy(np.ascontiguousarray(pairs, dtype=np.int32)).cuda()
    if n:
        check(lib().cmfw_exact_residues(
            ctypes.byref(desc), ctypes.c_void_p(d_in.data_ptr()), n, N, h,
            ctypes.c_void_p(d_primes.data_ptr()), K,
            ctypes.c_void_p(d_pairs.data_ptr()) if d_pairs is not None else None,
            ctypes.c_void_p(d_res.data_ptr()), ctypes.c_void_p(d_ok.data_ptr()), _stream_handle(None)))
    return d_res, d_ok, d_primes


def exact_reconstruct(d_res, d_ok, d_primes, n, K):
    """cmfw_exact_reconstruct over the first K primes of device residues
    (d_res [n, 3, 2, stride]): per (trajectory, depth) a status (0 fraction,
    1 zero denominator, 2 undetermined, 3 singular) and the fraction as a
    Python (numerator, denominator) pair where the status is 0."""
    torch = _torch()
    stride = int(d_res.shape[-1])
    W = lib().cmfw_exact_recon_words(int(K))
    T = 3 * n
    d_num = torch.zeros((max(T, 1), W), dtype=torch.int32, device="cuda")
    d_den = torch.zeros((max(T, 1), W), dtype=torch.int32, device="cuda")
    d_ln = torch.zeros(max(T, 1), dtype=torch.int32, device="cuda")
    d_ld = torch.zeros(max(T, 1), dtype=torch.int32, device="cuda")
    d_sg = torch.zeros(max(T, 1), dtype=torch.int8, device="cuda")
    d_st = torch.zeros(max(T, 1), dtype=torch.uint8, device="cuda")
    if n:
        check(lib().cmfw_exact_reconstruct(
            ctypes.c_void_p(d_res.data_ptr()), ctypes.c_void_p(d_ok.data_ptr()),
            ctypes.c_void_p(d_primes.data_ptr()), int(n), stride, int(K),
            ctypes.c_void_p(d_num.data_ptr()), ctypes.c_void_p(d_den.data_ptr()),
            ctypes.c_void_p(d_ln.data_ptr()), ctypes.c_void_p(d_ld.data_ptr()),
            ctypes.c_void_p(d_sg.data_ptr()), ctypes.c_void_p(d_st.data_ptr()), _stream_handle(None)))
    st = d_st[:T].cpu().numpy()
    ln, ld, sg = d_ln[:T].cpu().numpy(), d_ld[:T].cpu().numpy(), d_sg[:T].cpu().numpy()
    good = np.nonzero(st == 0)[0]
    fracs = [None] * T
    if len(good):
        gi = torch.from_numpy(good).cuda()
        nums = d_num[gi].cpu().numpy().view(np.uint32)
        dens = d_den[gi].cpu().numpy().view(np.uint32)
        for r, t in enumerate(good):
            num = int.from_bytes(nums[r, :ln[t]].tobytes(), "little")
            den = int.from_bytes(dens[r, :ld[t]].tobytes(), "little")
            fracs[t] = (-num if sg[t] < 0 else num, den)
    return st.reshape(n, 3), [fracs[3 * i:3 * i + 3] for i in range(n)]


def pipe_peak(pipe):
    """Measured FMA throughput (tera-ops/s, FMA = 2) of pipe 0 FP64, 1 FP32, 2 INT32."""
    v = ctypes.c_double(0)
    check(lib().cmfw_pipe_peak(int(pipe), ctypes.byref(v)))
    return v.value


def device_banner():
    buf = ctypes.create_string_buffer(512)
    check(lib().cmfw_device_banner(buf, 512))
    return buf.value.decode()


# ---- mixed batches ---------------------------------------------------------

def _descs_array(descs):
    arr = (Desc * len(descs))()
    for i, d in enumerate(descs):
        arr[i] = d
    return arr


def _variant_id(variant):
    if variant not in ("f64", "df64"):
        raise ValueError("mixed batches walk in f64 or df64")
    return VARIANTS[variant]


class MixedBatch:
    """A mixed batch resident on the device: records, per-trajectory
    (descriptor, depth) items, results and the workspace, ready to walk with
    cmfw_walk_mixed, to tune with cmfw_mixed_autotune, or to capture once
    into a CUDA graph (cmfw_mixed_graph_*) and replay."""

    def __init__(self, descs, records, items, h, variant="f64", with_status=False):
        torch = _torch()
        self.descs = list(descs)
        self.c_descs = _descs_array(self.descs)
        self.n = len(records)
        self.h = int(h)
        self.variant = _variant_id(variant)
        self.d_in = to_device(records)
        it = np.ascontiguousarray(items, dtype=MIXED_ITEM_DTYPE)
        self.d_items = torch.from_numpy(it.view(np.int32).reshape(-1)).cuda()
        self.d_out = out_buffer(self.n)
        nbytes = lib().cmfw_mixed_workspace_bytes(self.n, len(self.descs))
        self.d_ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
        self.d_status = torch.empty(max(self.n, 1), dtype=torch.uint8, device="cuda") if with_status else None
        self.launch = Launch()
        self.launch.d_workspace = self.d_ws.data_ptr()
        self.launch.workspace_bytes = nbytes
        self.launch.d_status = self.d_status.data_ptr() if with_status else None
        self._graph = None

    def _args(self):
        return (self.c_descs, len(self.descs), ctypes.c_void_p(self.d_in.data_ptr()),
                ctypes.c_void_p(self.d_items.data_ptr()), ctypes.c_void_p(self.d_out.data_ptr()),
                self.n, self.h, self.variant)

    def walk(self, tuning=None, stream=None):
        """Enqueue the mixed walk (no synchronisation)."""
        check(lib().cmfw_walk_mixed(*self._args(), ctypes.byref(tuning) if tuning is not None else None,
                                    ctypes.byref(self.launch), _stream_handle(stream)))

    def autotune(self, sample=0, stream=None):
        t = MixedTuning()
        check(lib().cmfw_mixed_autotune(*self._args(), ctypes.byref(self.launch), int(sample), ctypes.byref(t),
                                        _stream_handle(stream)))
        return t

    def capture(self, tuning=None):
        """Capture the whole walk into a CUDA graph (replaces a previous one)."""
        self.release()
        g = ctypes.c_void_p()
        check(lib().cmfw_mixed_graph_create(*self._args(), ctypes.byref(tuning) if tuning is not None else None,
                                            ctypes.byref(self.launch), ctypes.byref(g)))
        self._graph = g

    def replay(self, stream=None):
        if self._graph is None:
            raise RuntimeError("capture() first")
        check(lib().cmfw_mixed_graph_launch(self._graph, _stream_handle(stream)))

    def release(self):
        if self._graph is not None:
            lib().cmfw_mixed_graph_destroy(self._graph)
            self._graph = None

    def results(self):
        _torch().cuda.synchronize()
        out = records_from_device(self.d_out, self.n)
        if self.d_status is not None:
            return out, self.d_status[:self.n].cpu().numpy()
        return out

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def baseline_tuning():
    """The fixed baseline: one thread per sorted trajectory, 256-thread CTAs."""
    t = MixedTuning()
    t.persistent = 0
    return t


def walk_mixed(descs, records, items, h, variant="f64", tuning=None, with_status=False):
    """Walk a mixed batch and return its result records (and statuses)."""
    b = MixedBatch(descs, records, items, h, variant, with_status)
    b.walk(tuning)
    return b.results()
