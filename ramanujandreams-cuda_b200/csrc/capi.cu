// C ABI (include/cmfw.h): argument checks, scratch management, dispatch to
// the walk kernels, and the host-buffer convenience entry point.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <utility>

#include "cmfw.h"
#include "cmfw_internal.cuh"

namespace cmfw {
cudaError_t launch_walk_seq(const WalkArgs &W, bool ff, int block, cudaStream_t s);
cudaError_t launch_walk_chunked(const WalkArgs &W, bool ff, int threads, void *scratch, int prefix_steps,
                                cudaStream_t s, const HostGather *hg = nullptr);
size_t chunk_scratch_bytes(int dim, int n);
cudaError_t launch_walk_df64_compat(const WalkArgs &W, int block, cudaStream_t s);
cudaError_t launch_walk_rns(const WalkArgs &W, int n_primes, int trace_steps, uint32_t *trace_res,
                            int *trace_ok, int block, cudaStream_t s);
cudaError_t upload_compat_table();
cudaError_t launch_walk_exact(const cmfw_traj_in *in, int n_traj, int p, int q, int dim, int N, int h,
                              long long zn, long long zd, const uint32_t *primes, int K, const int *pairs,
                              uint32_t *res, uint8_t *prime_ok, cudaStream_t s);
}  // namespace cmfw

using namespace cmfw;

namespace {

thread_local std::string g_err;

cmfw_status set_err(cmfw_status s, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

cmfw_status cuda_err(cudaError_t e, const char *what) {
    return set_err(CMFW_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Library-owned scratch, one buffer per (device, stream): calls on one
// stream are ordered by the stream, calls on different streams never share.
struct Scratch {
    void *ptr = nullptr;
    size_t bytes = 0;
};
std::mutex g_mu;
std::map<std::pair<int, cudaStream_t>, Scratch> g_scratch;
std::map<int, bool> g_compat_ready;

cmfw_status library_scratch(size_t need, cudaStream_t s, void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_mu);
    Scratch &w = g_scratch[{dev, s}];
    if (w.bytes < need) {
        if (w.ptr) {
            e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return cuda_err(e, "cudaStreamSynchronize");
            cudaFree(w.ptr);
            w.ptr = nullptr;
            w.bytes = 0;
        }
        size_t grow = need + need / 4;
        e = cudaMalloc(&w.ptr, grow);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_err(CMFW_ENOMEM, "scratch allocation of %zu bytes failed", grow);
        }
        w.bytes = grow;
    }
    *out = w.ptr;
    return CMFW_OK;
}

cmfw_status ensure_compat_table() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_compat_ready[dev]) return CMFW_OK;
    e = upload_compat_table();
    if (e != cudaSuccess) return cuda_err(e, "compat modulus table upload");
    g_compat_ready[dev] = true;
    return CMFW_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device copies of cmfw_walk_host's records and its timing events, one set
// per calling thread and device, kept between calls (the call synchronises
// before returning).
struct Staging {
    void *in = nullptr, *out = nullptr;
    int cap = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // the call's timing events
    // chunked walks: the mapped pinned buffers that receive the survivors'
    // indices and results (h_cap entries)
    int *h_count = nullptr, *h_idx = nullptr;
    cmfw_traj_out *h_rec = nullptr;
    int h_cap = 0;
};
thread_local std::map<int, Staging> t_staging;

cudaError_t host_staging(int n, cmfw_traj_in **in, cmfw_traj_out **out, cudaEvent_t **ev) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    Staging &s = t_staging[dev];
    for (int i = 0; i < 4; ++i)
        if (!s.ev[i]) {
            e = cudaEventCreate(&s.ev[i]);
            if (e != cudaSuccess) return e;
        }
    *ev = s.ev;
    if (s.cap < n) {
        cudaFree(s.in);
        cudaFree(s.out);
        s.in = s.out = nullptr;
        s.cap = 0;
        e = cudaMalloc(&s.in, sizeof(cmfw_traj_in) * (size_t)n);
        if (e == cudaSuccess) e = cudaMalloc(&s.out, sizeof(cmfw_traj_out) * (size_t)n);
        if (e != cudaSuccess) return e;
        s.cap = n;
    }
    *in = (cmfw_traj_in *)s.in;
    *out = (cmfw_traj_out *)s.out;
    return cudaSuccess;
}

// The survivor buffers of cmfw_walk_host's chunked walks, for n results.
cudaError_t host_gather(int n, Staging **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    Staging &s = t_staging[dev];
    if (s.h_cap < n) {
        cudaFreeHost(s.h_count);
        cudaFreeHost(s.h_idx);
        cudaFreeHost(s.h_rec);
        s.h_count = s.h_idx = nullptr;
        s.h_rec = nullptr;
        s.h_cap = 0;
        e = cudaHostAlloc(&s.h_count, sizeof(int), cudaHostAllocMapped);
        if (e == cudaSuccess) e = cudaHostAlloc(&s.h_idx, sizeof(int) * (size_t)n, cudaHostAllocMapped);
        if (e == cudaSuccess) e = cudaHostAlloc(&s.h_rec, sizeof(cmfw_traj_out) * (size_t)n, cudaHostAllocMapped);
        if (e != cudaSuccess) return e;
        s.h_cap = n;
    }
    *out = &s;
    return cudaSuccess;
}

// Snapshot matrices and row exponents of every trajectory, followed by the
// chunked walk's survivor list and counter.
size_t snapshot_bytes(int dim, int n) {
    return align256((size_t)n * 3 * dim * dim * sizeof(double)) + align256((size_t)n * 3 * dim * sizeof(int)) +
           chunk_scratch_bytes(dim, n);
}

void *chunk_scratch(const WalkArgs &W) {
    return (char *)W.snap_e + align256((size_t)W.n_traj * 3 * W.dim * sizeof(int));
}

// Lattice steps walked one thread per trajectory before the chunked walk
// takes over the survivors: one is enough to drop the walks that fail at
// once (a singular first step), and the prefix is on every trajectory's
// critical path.
constexpr int kPrefixSteps = 1;

cudaError_t launch_float_walk(const WalkArgs &W, bool ff, int block, cudaStream_t s) {
    if (W.flags & CMFW_F_SEQUENTIAL) return launch_walk_seq(W, ff, block, s);
    return launch_walk_chunked(W, ff, block, chunk_scratch(W), kPrefixSteps, s);
}

cmfw_status check_walk_args(const cmfw_desc *desc, const void *d_in, const void *d_out, int n, int N,
                            int h) {
    if (!desc) return set_err(CMFW_EINVAL, "desc is NULL");
    cmfw_status s = cmfw_check_desc(desc);
    if (s != CMFW_OK) return s;
    if (n < 0) return set_err(CMFW_EINVAL, "n_traj = %d is negative", n);
    if (n > 0 && (!d_in || !d_out)) return set_err(CMFW_EINVAL, "NULL trajectory buffer");
    if (N > CMFW_MAX_DEPTH) return set_err(CMFW_EINVAL, "N = %d above CMFW_MAX_DEPTH", N);
    (void)h;
    return CMFW_OK;
}

cmfw_status prepare(const cmfw_desc *desc, const cmfw_traj_in *d_in, cmfw_traj_out *d_out, int n, int N,
                    int h, const cmfw_launch *launch, cudaStream_t s, WalkArgs &W) {
    cmfw_status st = check_walk_args(desc, d_in, d_out, n, N, h);
    if (st != CMFW_OK) return st;
    const size_t need = snapshot_bytes(desc->rank, n);
    void *ws = nullptr;
    if (launch && launch->d_workspace) {
        if (launch->workspace_bytes < need)
            return set_err(CMFW_EINVAL, "workspace of %zu bytes is below the %zu bytes needed",
                           launch->workspace_bytes, need);
        ws = launch->d_workspace;
    } else if (n > 0) {
        st = library_scratch(need, s, &ws);
        if (st != CMFW_OK) return st;
    }
    W.in = d_in;
    W.out = d_out;
    W.status = launch ? launch->d_status : nullptr;
    W.limit_src = launch ? launch->d_limit_src : nullptr;
    W.snap = (double *)ws;
    W.snap_e = (int *)((char *)ws + align256((size_t)n * 3 * desc->rank * desc->rank * sizeof(double)));
    W.n_traj = n;
    W.N = N;
    W.h = h;
    W.p = desc->p;
    W.q = desc->q;
    W.dim = desc->rank;
    W.z = desc->z;
    W.flags = launch ? launch->flags : 0;
    W.ev_main_start = launch ? launch->ev_main_start : nullptr;
    W.ev_main_stop = launch ? launch->ev_main_stop : nullptr;
    return CMFW_OK;
}

int block_of(const cmfw_launch *launch) { return launch ? launch->block_size : 0; }

}  // namespace

namespace cmfw {
// cmfw_last_error's message for entry points defined in other files.
cmfw_status record_error(cmfw_status s, const char *msg) { return set_err(s, "%s", msg); }
}  // namespace cmfw

extern "C" {

const char *cmfw_version(void) { return "cmfw 0.1.0 (sm_100a)"; }

const char *cmfw_last_error(void) { return g_err.c_str(); }

cmfw_desc cmfw_make_desc(int p, int q, double z) {
    cmfw_desc d;
    d.p = p;
    d.q = q;
    d.z = z;
    d.naxes = p + q;
    d.rank = (p > q + 1) ? p : q + 1;
    if (z == 1.0 && p == q + 1) d.rank -= 1;
    return d;
}

cmfw_status cmfw_check_desc(const cmfw_desc *d) {
    if (!d) return set_err(CMFW_EINVAL, "desc is NULL");
    if (d->p < 1 || d->p > 8) return set_err(CMFW_EINVAL, "p = %d outside 1..8", d->p);
    if (d->q < 0 || d->q > 7) return set_err(CMFW_EINVAL, "q = %d outside 0..7", d->q);
    if (d->naxes != d->p + d->q) return set_err(CMFW_EINVAL, "naxes = %d != p + q", d->naxes);
    if (d->rank < 2 || d->rank > CMFW_MAX_DIM) return set_err(CMFW_EINVAL, "rank = %d outside 2..8", d->rank);
    const int full = (d->p > d->q + 1) ? d->p : d->q + 1;
    if (d->rank != full && d->rank != full - 1)
        return set_err(CMFW_EINVAL, "rank = %d is neither max(p, q+1) nor one less", d->rank);
    if (!std::isfinite(d->z)) return set_err(CMFW_EINVAL, "z is not finite");
    return CMFW_OK;
}

size_t cmfw_walk_workspace_bytes(const cmfw_desc *desc, int n_traj) {
    if (!desc || n_traj < 0 || desc->rank < 1 || desc->rank > CMFW_MAX_DIM) return 0;
    return snapshot_bytes(desc->rank, n_traj);
}

cmfw_status cmfw_walk_f64(const cmfw_desc *desc, const cmfw_traj_in *d_in, cmfw_traj_out *d_out, int n,
                          int N, int h, const cmfw_launch *launch, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    WalkArgs W;
    cmfw_status st = prepare(desc, d_in, d_out, n, N, h, launch, s, W);
    if (st != CMFW_OK || n == 0) return st;
    cudaError_t e = launch_float_walk(W, false, block_of(launch), s);
    return e == cudaSuccess ? CMFW_OK : cuda_err(e, "f64 walk launch");
}

cmfw_status cmfw_walk_df64(const cmfw_desc *desc, const cmfw_traj_in *d_in, cmfw_traj_out *d_out, int n,
                           int N, int h, const cmfw_launch *launch, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    WalkArgs W;
    cmfw_status st = prepare(desc, d_in, d_out, n, N, h, launch, s, W);
    if (st != CMFW_OK || n == 0) return st;
    cudaError_t e = (W.flags & CMFW_F_DF64_COMPAT) ? launch_walk_df64_compat(W, block_of(launch), s)
                                                   : launch_float_walk(W, true, block_of(launch), s);
    return e == cudaSuccess ? CMFW_OK : cuda_err(e, "df64 walk launch");
}

cmfw_status cmfw_walk_rns(const cmfw_desc *desc, const cmfw_traj_in *d_in, cmfw_traj_out *d_out, int n,
                          int N, int h, int n_primes, const cmfw_launch *launch, void *stream) {
    if (n_primes < 1 || n_primes > CMFW_MAX_COMPAT_MODULI)
        return set_err(CMFW_EINVAL, "n_primes = %d outside 1..64", n_primes);
    cudaStream_t s = (cudaStream_t)stream;
    WalkArgs W;
    cmfw_status st = prepare(desc, d_in, d_out, n, N, h, launch, s, W);
    if (st != CMFW_OK || n == 0) return st;
    st = ensure_compat_table();
    if (st != CMFW_OK) return st;
    cudaError_t e = launch_walk_rns(W, n_primes, 0, nullptr, nullptr, block_of(launch), s);
    return e == cudaSuccess ? CMFW_OK : cuda_err(e, "rns walk launch");
}

cmfw_status cmfw_rns_trace(const cmfw_desc *desc, const cmfw_traj_in *d_in, int n, int N, int h,
                           int n_primes, int steps, int flags, uint32_t *d_res, int *d_ok, void *stream) {
    if (n_primes < 1 || n_primes > CMFW_MAX_COMPAT_MODULI)
        return set_err(CMFW_EINVAL, "n_primes = %d outside 1..64", n_primes);
    if (steps < 1) return set_err(CMFW_EINVAL, "steps = %d must be positive", steps);
    cmfw_status st = cmfw_check_desc(desc);
    if (st != CMFW_OK) return st;
    if (n < 0) return set_err(CMFW_EINVAL, "n_traj = %d is negative", n);
    if (n == 0) return CMFW_OK;
    if (!d_in || !d_res || !d_ok) return set_err(CMFW_EINVAL, "NULL buffer");
    st = ensure_compat_table();
    if (st != CMFW_OK) return st;
    WalkArgs W;
    memset(&W, 0, sizeof(W));
    W.in = d_in;
    W.n_traj = n;
    W.N = N;
    W.h = h;
    W.p = desc->p;
    W.q = desc->q;
    W.dim = desc->rank;
    W.z = desc->z;
    W.flags = flags;
    cudaError_t e = launch_walk_rns(W, n_primes, steps, d_res, d_ok, 0, (cudaStream_t)stream);
    return e == cudaSuccess ? CMFW_OK : cuda_err(e, "rns trace launch");
}

// z = zn / zd exactly (every finite double is a dyadic rational).
static bool split_dyadic(double z, long long *zn, long long *zd) {
    if (z == 0.0) { *zn = 0; *zd = 1; return true; }
    int e = 0;
    double mant = std::frexp(z, &e);        // z = mant * 2^e, 0.5 <= |mant| < 1
    long long M = (long long)std::ldexp(mant, 53);
    int E = e - 53;
    while ((M & 1LL) == 0) { M /= 2; ++E; }
    if (E >= 0) {
        long long mag = M < 0 ? -M : M;
        if (E > 62 || mag > (0x3fffffffffffffffLL >> E)) return false;
        *zn = M * (1LL << E);
        *zd = 1;
    } else {
        if (-E > 62) return false;
        *zn = M;
        *zd = 1LL << (-E);
    }
    return true;
}

cmfw_status cmfw_exact_residues(const cmfw_desc *desc, const cmfw_traj_in *d_in, int n, int N, int h,
                                const uint32_t *d_primes, int K, const int *d_pairs, uint32_t *d_res,
                                uint8_t *d_prime_ok, void *stream) {
    cmfw_status st = cmfw_check_desc(desc);
    if (st != CMFW_OK) return st;
    if (K < 1 || K > CMFW_MAX_EXACT_PRIMES) return set_err(CMFW_EINVAL, "K = %d outside 1..4096", K);
    if (n < 0) return set_err(CMFW_EINVAL, "n_traj = %d is negative", n);
    if (n == 0) return CMFW_OK;
    if (!d_in || !d_primes || !d_res || !d_prime_ok) return set_err(CMFW_EINVAL, "NULL buffer");
    long long zn, zd;
    if (!split_dyadic(desc->z, &zn, &zd)) return set_err(CMFW_EINVAL, "z = %g has no 62-bit dyadic form", desc->z);
    cudaError_t e = launch_walk_exact(d_in, n, desc->p, desc->q, desc->rank, N, h, zn, zd, d_primes, K, d_pairs,
                                      d_res, d_prime_ok, (cudaStream_t)stream);
    return e == cudaSuccess ? CMFW_OK : cuda_err(e, "exact walk launch");
}

cmfw_status cmfw_reference_inputs(int p, int q, int n, int mode, int use_zeta, cmfw_traj_in *h_out) {
    if (p < 1 || q < 0 || p + q > CMFW_MAX_AXES) return set_err(CMFW_EINVAL, "p = %d, q = %d out of range", p, q);
    if (n < 0) return set_err(CMFW_EINVAL, "n_traj = %d is negative", n);
    if (n > 0 && !h_out) return set_err(CMFW_EINVAL, "NULL output buffer");
    std::memset(h_out, 0, sizeof(cmfw_traj_in) * (size_t)n);
    // The reference's two generators write through pointers typed for
    // 128-byte positions and 16-int directions over an array of 192-byte
    // records; the bytes land where those strides put them, and that
    // placement is reproduced so that the same command line walks the same
    // trajectories.
    unsigned char *b = reinterpret_cast<unsigned char *>(h_out);
    const int naxes = p + q;
    auto put_f64 = [&](size_t off, double v) { std::memcpy(b + off, &v, 8); };
    auto put_i32 = [&](size_t off, int v) { std::memcpy(b + off, &v, 4); };
    auto get_i32 = [&](size_t off) { int v; std::memcpy(&v, b + off, 4); return v; };
    if (mode == 0) {
        if (use_zeta) {
            for (int i = 0; i < n; ++i)
                for (int a = 0; a < naxes; ++a) h_out[i].start[a] = a < p ? 1.0 : 2.0;
        } else {
            std::mt19937_64 rng(42);  // cmf_walk_f64.cu:61-71
            for (int i = 0; i < n; ++i)
                for (int a = 0; a < naxes; ++a) put_f64((size_t)i * 128 + 8 * a, (double)(2 + (int)(rng() % 19)));
        }
        for (int i = 0; i < n; ++i) {
            std::memset(h_out[i].dir, 0, sizeof(h_out[i].dir));
            h_out[i].dir[0] = 1;
        }
    } else {
        for (int i = 0; i < n; ++i)
            for (int a = 0; a < naxes; ++a)
                h_out[i].start[a] = use_zeta ? (a < p ? 1.0 : 2.0) : (a < p ? 2.0 : 3.0);
        std::mt19937_64 rng(42);  // cmf_walk_f64.cu:75-91
        const int dmax = 3;
        for (int i = 0; i < n; ++i) {
            const size_t base = (size_t)i * 64;
            for (int a = 0; a < naxes; ++a) put_i32(base + 4 * a, (int)(rng() % (2 * dmax + 1)) - dmax);
            bool all_zero = true;
            for (int a = 0; a < naxes; ++a)
                if (get_i32(base + 4 * a) != 0) { all_zero = false; break; }
            if (all_zero) put_i32(base, 1);
        }
    }
    return CMFW_OK;
}

void cmfw_mt64_fill(uint64_t seed, uint64_t *out, size_t n) {
    std::mt19937_64 rng(seed);
    for (size_t i = 0; i < n; ++i) out[i] = rng();
}

void cmfw_mt64_fill_at(uint64_t seed, uint64_t offset, uint64_t *out, size_t n) {
    std::mt19937_64 rng(seed);
    rng.discard(offset);
    for (size_t i = 0; i < n; ++i) out[i] = rng();
}

// cmfw_walk_host for the chunked f64 / df64 walks, the inputs already on
// their way to d_in: the host writes the filter's record for a dropped
// trajectory into every entry of h_out while the GPU walks, and the
// survivors' records, which the chunk kernel writes, come back through
// mapped pinned memory and are placed over them.
static cmfw_status walk_host_chunked(bool ff, const cmfw_desc *desc, cmfw_traj_out *h_out, cmfw_traj_in *d_in,
                                     cmfw_traj_out *d_out, int n, int N, int h, const cmfw_launch *launch,
                                     cudaEvent_t *ev, float *kernel_ms, float *total_ms) {
    Staging *S = nullptr;
    cudaError_t e = host_gather(n, &S);
    if (e != cudaSuccess) return set_err(CMFW_ENOMEM, "host buffers for %d results: %s", n, cudaGetErrorString(e));
    WalkArgs W;
    cmfw_status st = prepare(desc, d_in, d_out, n, N, h, launch, 0, W);
    if (st != CMFW_OK) return st;
    // Every trajectory the filter drops gets the same record (write_invalid:
    // NaN fields, valid 0; its status goes to launch->d_status), so the host
    // writes that record into h_out while the GPU walks, and only the
    // survivors' records come back, through mapped memory. No event sits
    // between the filter and the chunk kernel, which keeps the chunk
    // kernel's programmatic early launch.
    HostGather hg;
    e = cudaHostGetDevicePointer((void **)&hg.count, S->h_count, 0);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&hg.idx, S->h_idx, 0);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&hg.rec, S->h_rec, 0);
    if (e != cudaSuccess) return cuda_err(e, "mapped result buffers");
    e = launch_walk_chunked(W, ff, block_of(launch), chunk_scratch(W), kPrefixSteps, 0, &hg);
    if (e != cudaSuccess) return cuda_err(e, ff ? "df64 walk launch" : "f64 walk launch");
    cudaEventRecord(ev[2], 0);
    cudaEventRecord(ev[3], 0);
    cmfw_traj_out inv;
    inv.limit = inv.delta = inv.p = inv.q = inv.precision = inv.log_scale = std::numeric_limits<double>::quiet_NaN();
    inv.valid = 0;
    inv.n_limits = 0;
    for (int i = 0; i < n; ++i) h_out[i] = inv;
    e = cudaEventSynchronize(ev[3]);
    if (e != cudaSuccess && st == CMFW_OK) st = cuda_err(e, "walk execution");
    if (st != CMFW_OK) return st;
    const int c = *(volatile int *)S->h_count;
    for (int i = 0; i < c; ++i) h_out[S->h_idx[i]] = S->h_rec[i];
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, ev[1], ev[2]);
    cudaEventElapsedTime(&b, ev[0], ev[3]);
    if (kernel_ms) *kernel_ms = a;
    if (total_ms) *total_ms = b;
    return CMFW_OK;
}

cmfw_status cmfw_walk_host(cmfw_variant variant, const cmfw_desc *desc, const cmfw_traj_in *h_in,
                           cmfw_traj_out *h_out, int n, int N, int h, int n_primes, const cmfw_launch *launch,
                           float *kernel_ms, float *total_ms) {
    cmfw_status st = check_walk_args(desc, h_in, h_out, n, N, h);
    if (st != CMFW_OK) return st;
    if (variant == CMFW_VARIANT_RNS && (n_primes < 1 || n_primes > CMFW_MAX_COMPAT_MODULI))
        return set_err(CMFW_EINVAL, "n_primes = %d outside 1..64", n_primes);
    if (n == 0) {
        if (kernel_ms) *kernel_ms = 0.f;
        if (total_ms) *total_ms = 0.f;
        return CMFW_OK;
    }
    cmfw_traj_in *d_in = nullptr;
    cmfw_traj_out *d_out = nullptr;
    cudaEvent_t *ev = nullptr;
    cudaError_t e = host_staging(n, &d_in, &d_out, &ev);
    if (e != cudaSuccess) {
        st = set_err(CMFW_ENOMEM, "device buffers for %d trajectories: %s", n, cudaGetErrorString(e));
    } else {
        cudaEventRecord(ev[0], 0);
        e = cudaMemcpyAsync(d_in, h_in, sizeof(cmfw_traj_in) * (size_t)n, cudaMemcpyHostToDevice, 0);
        if (e != cudaSuccess) st = cuda_err(e, "input copy");
        cudaEventRecord(ev[1], 0);
        const int flags = launch ? launch->flags : 0;
        const bool chunked = (variant == CMFW_VARIANT_F64 || variant == CMFW_VARIANT_DF64) &&
                             !(flags & CMFW_F_SEQUENTIAL) &&
                             !(variant == CMFW_VARIANT_DF64 && (flags & CMFW_F_DF64_COMPAT));
        if (st == CMFW_OK && chunked)
            return walk_host_chunked(variant == CMFW_VARIANT_DF64, desc, h_out, d_in, d_out, n, N, h, launch, ev,
                                     kernel_ms, total_ms);
        if (st == CMFW_OK) {
            if (variant == CMFW_VARIANT_F64) st = cmfw_walk_f64(desc, d_in, d_out, n, N, h, launch, nullptr);
            else if (variant == CMFW_VARIANT_DF64) st = cmfw_walk_df64(desc, d_in, d_out, n, N, h, launch, nullptr);
            else st = cmfw_walk_rns(desc, d_in, d_out, n, N, h, n_primes, launch, nullptr);
        }
        cudaEventRecord(ev[2], 0);
        if (st == CMFW_OK) {
            e = cudaMemcpyAsync(h_out, d_out, sizeof(cmfw_traj_out) * (size_t)n, cudaMemcpyDeviceToHost, 0);
            if (e != cudaSuccess) st = cuda_err(e, "result copy");
        }
        cudaEventRecord(ev[3], 0);
        e = cudaEventSynchronize(ev[3]);
        if (e != cudaSuccess && st == CMFW_OK) st = cuda_err(e, "walk execution");
        if (st == CMFW_OK) {
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ev[1], ev[2]);
            cudaEventElapsedTime(&b, ev[0], ev[3]);
            if (kernel_ms) *kernel_ms = a;
            if (total_ms) *total_ms = b;
        }
    }
    return st;
}

cmfw_status cmfw_device_banner(char *buf, size_t size) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDeviceProperties");
    snprintf(buf, size, "GPU: %s (SM %d.%d, %d MPs, %.1f GB global mem)", prop.name, prop.major, prop.minor,
             prop.multiProcessorCount, prop.totalGlobalMem / 1e9);
    return CMFW_OK;
}

cmfw_status cmfw_device_meminfo(size_t *free_bytes, size_t *total_bytes) {
    size_t f = 0, t = 0;
    cudaError_t e = cudaMemGetInfo(&f, &t);
    if (e != cudaSuccess) return cuda_err(e, "cudaMemGetInfo");
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return CMFW_OK;
}

}  // extern "C"
