"""ctypes bindings for the CPU checkers (test infrastructure only)."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

IN_DTYPE = np.dtype([("dir", "<i4", 16), ("start", "<f8", 16)])
OUT_DTYPE = np.dtype([("limit", "<f8"), ("delta", "<f8"), ("p", "<f8"), ("q", "<f8"),
                      ("precision", "<f8"), ("log_scale", "<f8"), ("valid", "<i4"),
                      ("n_limits", "<i4")])
OUT_F64_DTYPE = np.dtype(OUT_DTYPE.descr + [("elapsed_ms", "<f8")])
assert IN_DTYPE.itemsize == 192 and OUT_DTYPE.itemsize == 56 and OUT_F64_DTYPE.itemsize == 64

_c_int, _c_dbl, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p


def build(with_ref=None, ref_root=None):
    """Compile liboracle.so, and the reference checkers (oracle/_ref) from the
    reference checkout named by ref_root or CMFW_REF_ROOT when it exists."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref_root = ref_root or os.environ.get("CMFW_REF_ROOT")
    if with_ref is None:
        with_ref = bool(ref_root) and os.path.isdir(os.path.join(ref_root, "cuda"))
    if with_ref:
        if not ref_root:
            raise RuntimeError("CMFW_REF_ROOT must name the reference checkout to build oracle/_ref")
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={ref_root}"], check=True)


_lib = None


def _oracle():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            build(with_ref=False)
        lib = ctypes.CDLL(ORACLE_LIB)
        walk_args = [_c_int, _c_int, _c_dbl, _c_int, _c_int, _vp, _vp, _c_int]
        lib.orc_walk_f64.argtypes = walk_args + [_c_int, _c_int]
        lib.orc_walk_f64_src.argtypes = walk_args + [_c_int, _c_int, _vp]
        lib.orc_exact_residues.argtypes = [_c_int, _c_int, ctypes.c_longlong, ctypes.c_longlong, _c_int,
                                           _c_int, _vp, _c_int, _vp, _c_int, _vp, _vp, _vp, _c_int]
        lib.orc_walk_df64.argtypes = walk_args + [_c_int, _c_int]
        lib.orc_walk_rns.argtypes = walk_args + [_c_int, _c_int, _c_int]
        lib.orc_make_inputs.argtypes = [_c_int, _c_int, _c_int, _c_int, _c_int, _vp]
        lib.orc_mt64_stream.argtypes = [ctypes.c_uint64, _vp, _c_int]
        lib.orc_f64_snapshots.argtypes = [_c_int, _c_int, _c_dbl, _c_int, _c_int, _vp, _vp,
                                          _c_int, _vp, _vp]
        lib.orc_rns_trace.argtypes = [_c_int, _c_int, _c_dbl, _c_int, _c_int, _vp, _vp, _c_int,
                                      _c_int, _c_int, _vp, _vp]
        lib.orc_rns_moduli.argtypes = [_vp, _c_int]
        lib.orc_column.argtypes = [_vp, _c_dbl, _c_int, _c_int, _c_int, _vp, _c_int]
        _lib = lib
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_vp)


def make_inputs(p, q, n, mode, use_zeta):
    """Input records as the reference's run_benchmark() builds them."""
    buf = np.zeros(n, dtype=IN_DTYPE)
    _oracle().orc_make_inputs(p, q, n, mode, int(use_zeta), _ptr(buf))
    return buf


def mt64_stream(seed, n):
    out = np.zeros(n, dtype=np.uint64)
    _oracle().orc_mt64_stream(seed, _ptr(out), n)
    return out


def walk(variant, p, q, z, N, h, inputs, n_primes=8, fused=False, threads=0):
    """Run the oracle walk; variant in {"f64", "df64", "rns"}."""
    inputs = np.ascontiguousarray(inputs, dtype=IN_DTYPE)
    n = len(inputs)
    lib = _oracle()
    if variant == "f64":
        out = np.zeros(n, dtype=OUT_F64_DTYPE)
        lib.orc_walk_f64(p, q, z, N, h, _ptr(inputs), _ptr(out), n, int(fused), threads)
    elif variant == "df64":
        out = np.zeros(n, dtype=OUT_DTYPE)
        lib.orc_walk_df64(p, q, z, N, h, _ptr(inputs), _ptr(out), n, int(fused), threads)
    elif variant == "rns":
        out = np.zeros(n, dtype=OUT_DTYPE)
        lib.orc_walk_rns(p, q, z, N, h, _ptr(inputs), _ptr(out), n, n_primes, int(fused), threads)
    else:
        raise ValueError(variant)
    return out


def walk_f64_src(p, q, z, N, h, inputs, fused=False, threads=0):
    """The f64 oracle walk and, per row, the source of its limit: (method
    << 12) | (i << 8) | (j << 4) | c for the ratio M[i][c] / M[j][c] chosen
    by the reference's reduction (method 1 = Aitken, 0 = raw), -1 when the
    row has no limit."""
    inputs = np.ascontiguousarray(inputs, dtype=IN_DTYPE)
    n = len(inputs)
    out = np.zeros(n, dtype=OUT_F64_DTYPE)
    src = np.full(n, -1, dtype=np.int32)
    _oracle().orc_walk_f64_src(p, q, z, N, h, _ptr(inputs), _ptr(out), n, int(fused), threads, _ptr(src))
    return out, src


def exact_residues(p, q, zn, zd, N, h, inputs, primes, pairs=None, threads=0):
    """Exact walk modulo each prime (odd, below 2^31): residues of the
    entries (i, c) and (j, c) of the walk matrix at depths N-2h, N-h, N as
    an array [n, 3, 2, K], and a per-prime usability mask [n, K]."""
    inputs = np.ascontiguousarray(inputs, dtype=IN_DTYPE)
    primes = np.ascontiguousarray(primes, dtype=np.uint32)
    n, K = len(inputs), len(primes)
    res = np.zeros((n, 3, 2, K), dtype=np.uint32)
    ok = np.zeros((n, K), dtype=np.uint8)
    pr = None
    if pairs is not None:
        pr = np.ascontiguousarray(pairs, dtype=np.int32)
        assert len(pr) == n
    if n and K:
        _oracle().orc_exact_residues(p, q, int(zn), int(zd), N, h, _ptr(inputs), n, _ptr(primes), K,
                                     None if pr is None else _ptr(pr), _ptr(res), _ptr(ok), threads)
    return res, ok.astype(bool)


def _dir_start(dir_, start):
    d = np.zeros(16, dtype=np.int32)
    s = np.zeros(16, dtype=np.float64)
    d[:len(dir_)] = dir_
    s[:len(start)] = start
    return d, s


def f64_snapshots(p, q, z, N, h, dir_, start, fused=False):
    d, s = _dir_start(dir_, start)
    m = np.zeros((3, 8, 8))
    ls = np.zeros(3)
    ok = _oracle().orc_f64_snapshots(p, q, z, N, h, _ptr(d), _ptr(s), int(fused), _ptr(m), _ptr(ls))
    return bool(ok), m, ls


def rns_trace(p, q, z, N, h, dir_, start, n_primes, steps, rank, fused=False):
    d, s = _dir_start(dir_, start)
    out = np.zeros((n_primes, rank, rank), dtype=np.uint32)
    ls = ctypes.c_double(0.0)
    ok = _oracle().orc_rns_trace(p, q, z, N, h, _ptr(d), _ptr(s), n_primes, steps, int(fused),
                                 _ptr(out), ctypes.byref(ls))
    return bool(ok), out, ls.value


def rns_moduli(n=64):
    out = np.zeros(n, dtype=np.uint32)
    _oracle().orc_rns_moduli(_ptr(out), n)
    return out


def column(pos, z, dim, p, q, fused=False):
    pv = np.zeros(16)
    pv[:len(pos)] = pos
    col = np.zeros(8)
    ok = _oracle().orc_column(_ptr(pv), z, dim, p, q, _ptr(col), int(fused))
    return bool(ok), col[:dim]


# ---------------------------------------------------------------------------
# The reference's own kernel bodies, compiled for the host (oracle/_ref).
# ---------------------------------------------------------------------------
_ref_libs = {}


def _ref_path(variant, fused):
    return os.path.join(REF_DIR, f"libref_{variant}{'_fma' if fused else ''}.so")


def have_ref(variant="f64", fused=False):
    return os.path.exists(_ref_path(variant, fused))


def _ref(variant, fused=False):
    key = (variant, fused)
    if key not in _ref_libs:
        lib = ctypes.CDLL(_ref_path(variant, fused))
        pre = f"ref_{variant}_"
        getattr(lib, pre + "walk").argtypes = [_c_int, _c_int, _c_dbl, _c_int, _c_int, _vp, _vp,
                                               _c_int, _c_int, _c_int]
        getattr(lib, pre + "make_inputs").argtypes = [_c_int, _c_int, _c_int, _c_int, _c_int, _vp]
        if variant == "f64":
            lib.ref_f64_snapshots.argtypes = [_c_int, _c_int, _c_dbl, _c_int, _c_int, _vp, _vp,
                                              _vp, _vp]
        if variant == "rns":
            lib.ref_rns_trace.argtypes = [_c_int, _c_int, _c_dbl, _c_int, _c_int, _vp, _vp,
                                          _c_int, _c_int, _vp, _vp]
            lib.ref_rns_primes.argtypes = [_vp, _c_int]
        _ref_libs[key] = lib
    return _ref_libs[key]


def ref_make_inputs(p, q, n, mode, use_zeta, variant="f64"):
    buf = np.zeros(n, dtype=IN_DTYPE)
    getattr(_ref(variant), f"ref_{variant}_make_inputs")(p, q, n, mode, int(use_zeta), _ptr(buf))
    return buf


def ref_walk(variant, p, q, z, N, h, inputs, n_primes=8, fused=False, threads=0):
    inputs = np.ascontiguousarray(inputs, dtype=IN_DTYPE)
    n = len(inputs)
    out = np.zeros(n, dtype=OUT_F64_DTYPE if variant == "f64" else OUT_DTYPE)
    getattr(_ref(variant, fused), f"ref_{variant}_walk")(p, q, z, N, h, _ptr(inputs), _ptr(out),
                                                         n, n_primes, threads)
    return out


def ref_f64_snapshots(p, q, z, N, h, dir_, start, fused=False):
    d, s = _dir_start(dir_, start)
    m = np.zeros((3, 8, 8))
    ls = np.zeros(3)
    ok = _ref("f64", fused).ref_f64_snapshots(p, q, z, N, h, _ptr(d), _ptr(s), _ptr(m), _ptr(ls))
    return bool(ok), m, ls


def ref_rns_trace(p, q, z, N, h, dir_, start, n_primes, steps, rank, fused=False):
    d, s = _dir_start(dir_, start)
    out = np.zeros((n_primes, rank, rank), dtype=np.uint32)
    ls = ctypes.c_double(0.0)
    ok = _ref("rns", fused).ref_rns_trace(p, q, z, N, h, _ptr(d), _ptr(s), n_primes, steps,
                                          _ptr(out), ctypes.byref(ls))
    return bool(ok), out, ls.value


def ref_rns_moduli(n=64):
    out = np.zeros(n, dtype=np.uint32)
    _ref("rns").ref_rns_primes(_ptr(out), n)
    return out


# ---------------------------------------------------------------------------
# The reference's own CUDA kernels built for sm_100a (oracle/_ref, comparison
# arm of the benchmark).
# ---------------------------------------------------------------------------
def have_ref_gpu(variant="f64"):
    return os.path.exists(os.path.join(REF_DIR, f"libref_gpu_{variant}.so"))


def ref_gpu_launch(variant, p, q, z, N, h, d_in, d_out, n, block=0, stream=0, n_primes=8):
    """Launch the reference kernel walk_kernel_<variant> on device buffers
    (integer device addresses of n reference input / result records) on
    `stream`; block 0 = the reference's default (256, RNS 128)."""
    key = ("gpu", variant)
    if key not in _ref_libs:
        lib = ctypes.CDLL(os.path.join(REF_DIR, f"libref_gpu_{variant}.so"))
        args = [_vp, _vp, _c_int, _c_int, _c_dbl, _c_int, _c_int, _c_int, _c_int]
        fn = getattr(lib, f"ref_gpu_{variant}_launch")
        fn.argtypes = args + ([_c_int] if variant == "rns" else []) + [_vp]
        _ref_libs[key] = lib
    fn = getattr(_ref_libs[key], f"ref_gpu_{variant}_launch")
    block = block or (128 if variant == "rns" else 256)
    extra = [n_primes] if variant == "rns" else []
    rc = fn(_vp(d_in), _vp(d_out), p, q, z, N, h, n, block, *extra, _vp(stream))
    if rc != 0:
        raise RuntimeError(f"reference {variant} kernel launch failed: CUDA error {rc}")
