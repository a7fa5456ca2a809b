// Mixed batches: trajectories of different CMF families (p, q, z, rank) and
// different depths N walked in one enqueue -- and, through
// cmfw_mixed_graph_*, one CUDA graph launch.
//
// The reference runs one family at one depth per program invocation
// (cmf_walk_f64.cu:156-305); a mixed batch of 10^6 trajectories with N
// log-uniform in 200..5000 is dominated by load balance: a plain grid of one
// thread per trajectory mixes 200-step and 5000-step walks in every warp and
// finishes with the GPU mostly idle. The pipeline here:
//
//  1. keys:    per trajectory, its family and a cost bucket from
//              N * sum|dir| (axis steps), counted into a histogram
//              (family-major, cost descending);
//  2. scan:    one CTA turns the histogram into segment offsets;
//  3. scatter: trajectory indices into cost-sorted order per family;
//  4. walk:    per family, a persistent kernel (grid = SMs x resident CTAs)
//              whose warps take `grab` consecutive sorted trajectories at a
//              time from the family's queue (an atomic counter): neighbours
//              in a warp have similar depth and the longest walks start
//              first, so the tail is short; or a plain grid of one
//              trajectory per thread in cost order (tile grab 0).
//  Optional (tuning->prescan): before 4, a persistent scan follows each
//  trajectory through its N steps with the position-only singularity tests
//  (no matrix), writes the failures' results at once and compacts the
//  survivors for the walk. On the benchmark mix it costs more than it saves
//  (the tests are over half a step's work at small ranks, and survivors pay
//  for both), so it is off by default.
//
// The walk of one trajectory is the sequential kernel's (walk_seq.cuh) in the
// launch's arithmetic (FP64, or float-float on the FP32 pipe with the FP64
// finalisation of the snapshot reduction). Block size, grab and resident
// CTAs per SM are per family (cmfw_mixed_tuning), chosen by
// cmfw_mixed_autotune from timed runs on a sample of the batch. With
// tuning->persistent = 0 the walk is the baseline: one thread per sorted
// trajectory, a plain grid of 256-thread CTAs.
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <vector>

#include "cmfw.h"
#include "walk_seq.cuh"

namespace cmfw {
cmfw_status record_error(cmfw_status s, const char *msg);

constexpr int kCostBuckets = 64;

struct MixedArgs {
    WalkArgs w;                    // in, out, status, limit_src, h
    const cmfw_mixed_item *items;  // per trajectory: desc index, depth
    const int *order;              // trajectory indices, sorted
    const int *begin;              // n_descs + 1 offsets of each family in order
    int *next;                     // n_descs queue heads (start at zero)
    const int *seg_len;            // optional: family lengths (else begin[f+1] - begin[f])
    int *alive;                    // survivors of the scan, at each family's offset
    int *alive_count;              // n_descs
    int grab;                      // trajectories a warp takes per queue access
    cmfw_desc descs[CMFW_MAX_MIXED_DESCS];
    int n_descs;
};

__device__ __forceinline__ int cost_bucket(long long cost) {
    // descending: the most expensive trajectories get bucket 0
    if (cost < 1) cost = 1;
    const int lg = 63 - __clzll(cost);                                // floor(log2)
    const int half = (int)((cost >> (lg > 0 ? lg - 1 : 0)) & 1);      // next bit
    const int b = 2 * lg + (lg > 0 ? half : 0);
    return max(0, kCostBuckets - 1 - min(b, kCostBuckets - 1));
}

__global__ void mixed_keys_kernel(MixedArgs M, int *keys, int *hist) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M.w.n_traj) return;
    const cmfw_mixed_item it = M.items[t];
    if (it.desc < 0 || it.desc >= M.n_descs) {
        write_invalid(M.w, t, CMFW_TRAJ_BAD_FAMILY);
        keys[t] = -1;
        return;
    }
    const int naxes = M.descs[it.desc].naxes;
    long long steps = 0;
    for (int a = 0; a < naxes && a < CMFW_MAX_AXES; ++a) steps += abs(M.w.in[t].dir[a]);
    const long long cost = (long long)max(it.N, 1) * max(steps, 1LL);
    const int key = it.desc * kCostBuckets + cost_bucket(cost);
    keys[t] = key;
    atomicAdd(&hist[key], 1);
}

// One CTA of 1024 threads: exclusive scan of n_descs * 64 counts (<= 1024).
__global__ void __launch_bounds__(1024) mixed_scan_kernel(const int *hist, int *cursor, int *begin, int n_keys,
                                                          int n_descs) {
    __shared__ int s[1024];
    const int i = threadIdx.x;
    const int v = i < n_keys ? hist[i] : 0;
    s[i] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int add = i >= off ? s[i - off] : 0;
        __syncthreads();
        s[i] += add;
        __syncthreads();
    }
    if (i < n_keys) cursor[i] = s[i] - v;
    if (i <= n_descs) {
        const int k = i * kCostBuckets;
        begin[i] = k < n_keys ? s[k] - hist[k] : s[n_keys - 1];
    }
}

__global__ void mixed_scatter_kernel(const int *keys, int *cursor, int *order, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int k = keys[t];
    if (k < 0) return;
    order[atomicAdd(&cursor[k], 1)] = t;
}

// Walks family `fam` of the batch: persistent (queue) or one thread per
// sorted trajectory.
template <int P_, int Q_, int DIM, class A>
__global__ void __launch_bounds__(256) walk_mixed_kernel(MixedArgs M, int fam, int persistent) {
    WalkArgs W = M.w;
    W.p = M.descs[fam].p;
    W.q = M.descs[fam].q;
    W.dim = M.descs[fam].rank;
    W.z = M.descs[fam].z;
    double snap[3 * DIM * DIM];
    int snap_e[3 * DIM];
    const int lo = M.begin[fam];
    const int len = M.seg_len ? M.seg_len[fam] : M.begin[fam + 1] - lo;
    if (!persistent) {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i < len) {
            const int t = M.order[lo + i];
            walk_seq_one<P_, Q_, DIM, A>(W, t, M.items[t].N, snap, snap_e);
        }
        return;
    }
    const int lane = threadIdx.x & 31;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&M.next[fam], M.grab);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= len) break;
        for (int k = lane; k < M.grab; k += 32) {
            const int i = base + k;
            if (i < len) {
                const int t = M.order[lo + i];
                walk_seq_one<P_, Q_, DIM, A>(W, t, M.items[t].N, snap, snap_e);
            }
        }
    }
}

// The singularity scan of family `fam`: each trajectory of its sorted
// segment is followed through steps 1..N with the position-only tests; a
// failure is written as the trajectory's result right away, a survivor is
// appended to the family's part of M.alive for the walk.
template <int P_, int Q_, int DIM>
__global__ void __launch_bounds__(256) scan_mixed_kernel(MixedArgs M, int fam) {
    WalkArgs W = M.w;
    W.p = M.descs[fam].p;
    W.q = M.descs[fam].q;
    W.dim = M.descs[fam].rank;
    W.z = M.descs[fam].z;
    const int lo = M.begin[fam];
    const int len = M.begin[fam + 1] - lo;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&M.next[fam], 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= len) break;
        const int i = base + lane;
        if (i < len) {
            const int t = M.order[lo + i];
            const int st = scan_failure<P_, Q_, DIM>(W, t, M.items[t].N);
            if (st != CMFW_TRAJ_OK) write_invalid(W, t, st);
            else M.alive[lo + atomicAdd(&M.alive_count[fam], 1)] = t;
        }
    }
}

typedef void (*scan_kernel_t)(MixedArgs, int);

static scan_kernel_t pick_scan(int p, int q, int dim) {
#define CMFW_CASE(P, Q, D) \
    if (p == P && q == Q && dim == D) return scan_mixed_kernel<P, Q, D>;
    CMFW_FAMILY_CASES
#undef CMFW_CASE
    switch (dim) {
        case 2: return scan_mixed_kernel<0, 0, 2>;
        case 3: return scan_mixed_kernel<0, 0, 3>;
        case 4: return scan_mixed_kernel<0, 0, 4>;
        case 5: return scan_mixed_kernel<0, 0, 5>;
        case 6: return scan_mixed_kernel<0, 0, 6>;
        case 7: return scan_mixed_kernel<0, 0, 7>;
        case 8: return scan_mixed_kernel<0, 0, 8>;
    }
    return nullptr;
}

typedef void (*mixed_kernel_t)(MixedArgs, int, int);

template <class A>
static mixed_kernel_t pick_mixed(int p, int q, int dim) {
#define CMFW_CASE(P, Q, D) \
    if (p == P && q == Q && dim == D) return walk_mixed_kernel<P, Q, D, A>;
    CMFW_FAMILY_CASES
#undef CMFW_CASE
    switch (dim) {
        case 2: return walk_mixed_kernel<0, 0, 2, A>;
        case 3: return walk_mixed_kernel<0, 0, 3, A>;
        case 4: return walk_mixed_kernel<0, 0, 4, A>;
        case 5: return walk_mixed_kernel<0, 0, 5, A>;
        case 6: return walk_mixed_kernel<0, 0, 6, A>;
        case 7: return walk_mixed_kernel<0, 0, 7, A>;
        case 8: return walk_mixed_kernel<0, 0, 8, A>;
    }
    return nullptr;
}

static mixed_kernel_t pick_mixed_variant(int variant, const cmfw_desc &d) {
    return variant == CMFW_VARIANT_DF64 ? pick_mixed<ArithFF>(d.p, d.q, d.rank)
                                        : pick_mixed<ArithF64>(d.p, d.q, d.rank);
}

// Workspace: histogram and cursors (n_descs * 64 ints each), begin
// (n_descs + 1), queue heads (n_descs), keys (n), order (n).
struct MixedLayout {
    int *hist, *cursor, *begin, *next, *next2, *alive_count, *keys, *order, *alive;
    size_t small_bytes;  // what must be zeroed before each walk
};

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t mixed_small_bytes() {
    return al256(sizeof(int) * (2 * CMFW_MAX_MIXED_DESCS * kCostBuckets + 4 * (CMFW_MAX_MIXED_DESCS + 1)));
}

static size_t mixed_ws_bytes(int n, int n_descs) {
    (void)n_descs;
    return mixed_small_bytes() + 3 * al256(sizeof(int) * (size_t)(n > 0 ? n : 1));
}

static MixedLayout mixed_layout(void *ws, int n) {
    MixedLayout L;
    int *p = (int *)ws;
    L.hist = p;
    L.cursor = p + CMFW_MAX_MIXED_DESCS * kCostBuckets;
    L.begin = L.cursor + CMFW_MAX_MIXED_DESCS * kCostBuckets;
    L.next = L.begin + CMFW_MAX_MIXED_DESCS + 1;
    L.next2 = L.next + CMFW_MAX_MIXED_DESCS + 1;
    L.alive_count = L.next2 + CMFW_MAX_MIXED_DESCS + 1;
    L.small_bytes = mixed_small_bytes();
    const size_t arr = al256(sizeof(int) * (size_t)(n > 0 ? n : 1));
    char *q = (char *)ws + L.small_bytes;
    L.keys = (int *)q;
    L.order = (int *)(q + arr);
    L.alive = (int *)(q + 2 * arr);
    return L;
}

static void default_tile(cmfw_mixed_tile &t) {
    t.block_size = 128;
    t.grab = 32;
    t.ctas_per_sm = 0;
}

static int sm_count() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// Resident CTAs of `k` per SM at `block` threads (at least 1).
static int resident_ctas(mixed_kernel_t k, int block) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void *)k, block, 0) != cudaSuccess || nb < 1)
        nb = 1;
    return nb;
}

// The sort (stages 1-3); the workspace's small part must be zero.
static cudaError_t enqueue_sort(const MixedArgs &M, const MixedLayout &L, cudaStream_t s) {
    const int n = M.w.n_traj;
    cudaError_t e = cudaMemsetAsync(L.hist, 0, L.small_bytes, s);
    if (e != cudaSuccess) return e;
    mixed_keys_kernel<<<(n + 255) / 256, 256, 0, s>>>(M, L.keys, L.hist);
    mixed_scan_kernel<<<1, 1024, 0, s>>>(L.hist, L.cursor, L.begin, M.n_descs * kCostBuckets, M.n_descs);
    mixed_scatter_kernel<<<(n + 255) / 256, 256, 0, s>>>(L.keys, L.cursor, L.order, n);
    return cudaGetLastError();
}

// One family's walk: a plain grid of one trajectory per thread (baseline,
// or a tile with grab 0), or the persistent queue of the tile.
static cudaError_t enqueue_family(const MixedArgs &M, int f, int variant, const cmfw_mixed_tile &tile,
                                  int persistent, cudaStream_t s) {
    mixed_kernel_t k = pick_mixed_variant(variant, M.descs[f]);
    if (!k) return cudaErrorInvalidValue;
    MixedArgs Mf = M;
    int block = tile.block_size;
    if (block != 64 && block != 128 && block != 256) block = 128;
    if (!persistent || tile.grab == 0) {
        if (!persistent) block = 256;
        const int n = M.w.n_traj;
        k<<<(n + block - 1) / block, block, 0, s>>>(Mf, f, 0);
        return cudaGetLastError();
    }
    Mf.grab = (tile.grab >= 32 && tile.grab % 32 == 0) ? tile.grab : 32;
    int per_sm = resident_ctas(k, block);
    if (tile.ctas_per_sm > 0 && tile.ctas_per_sm < per_sm) per_sm = tile.ctas_per_sm;
    k<<<sm_count() * per_sm, block, 0, s>>>(Mf, f, 1);
    return cudaGetLastError();
}

static cmfw_status check_mixed(const cmfw_desc *descs, int n_descs, int n, int h, int variant) {
    if (!descs || n_descs < 1 || n_descs > CMFW_MAX_MIXED_DESCS)
        return record_error(CMFW_EINVAL, "n_descs must be 1..16 with a descriptor array");
    for (int i = 0; i < n_descs; ++i) {
        cmfw_status s = cmfw_check_desc(&descs[i]);
        if (s != CMFW_OK) return s;
    }
    if (n < 0) return record_error(CMFW_EINVAL, "n_traj is negative");
    if (h <= 0) return record_error(CMFW_EINVAL, "h must be positive");
    if (variant != CMFW_VARIANT_F64 && variant != CMFW_VARIANT_DF64)
        return record_error(CMFW_EINVAL, "mixed batches walk in f64 or df64");
    return CMFW_OK;
}

static MixedArgs make_args(const cmfw_desc *descs, int n_descs, const cmfw_traj_in *d_in,
                           const cmfw_mixed_item *d_items, cmfw_traj_out *d_out, int n, int h,
                           const cmfw_launch *launch, const MixedLayout &L) {
    MixedArgs M;
    memset(&M, 0, sizeof(M));
    M.w.in = d_in;
    M.w.out = d_out;
    M.w.status = launch ? launch->d_status : nullptr;
    M.w.limit_src = launch ? launch->d_limit_src : nullptr;
    M.w.n_traj = n;
    M.w.h = h;
    M.w.flags = launch ? launch->flags : 0;
    M.items = d_items;
    M.order = L.order;
    M.begin = L.begin;
    M.next = L.next;
    M.seg_len = nullptr;
    M.alive = L.alive;
    M.alive_count = L.alive_count;
    M.grab = 32;
    for (int i = 0; i < n_descs; ++i) M.descs[i] = descs[i];
    M.n_descs = n_descs;
    return M;
}

// One family on stream s: the singularity scan (persistent, cost-sorted
// queue) and the walk of its survivors only (prescan), or the walk of
// every trajectory.
static cudaError_t enqueue_family_scan_walk(const MixedArgs &M, const MixedLayout &L, int f, int variant,
                                            const cmfw_mixed_tuning &tune, bool prescan, cudaStream_t s) {
    if (!prescan) return enqueue_family(M, f, variant, tune.tile[f], tune.persistent, s);
    scan_kernel_t k = pick_scan(M.descs[f].p, M.descs[f].q, M.descs[f].rank);
    if (!k) return cudaErrorInvalidValue;
    MixedArgs Ms = M;
    Ms.next = L.next2;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void *)k, 256, 0) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 1;
    }
    k<<<sm_count() * nb, 256, 0, s>>>(Ms, f);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    MixedArgs Mw = M;
    Mw.order = L.alive;
    Mw.seg_len = L.alive_count;
    return enqueue_family(Mw, f, variant, tune.tile[f], 1, s);
}

// Streams and events on which the families' walks run side by side: a
// family's walk ends with its longest trajectories on a few SMs, and the
// other families' CTAs fill the rest. One set per host thread and device,
// kept for the process (the enqueue is also captured into graphs, where
// the fork and join become parallel branches).
struct ForkStreams {
    cudaStream_t s[CMFW_MAX_MIXED_DESCS] = {};
    cudaEvent_t start = nullptr, done[CMFW_MAX_MIXED_DESCS] = {};
    bool ready = false;
};
static thread_local ForkStreams t_fork[16];

static cudaError_t fork_streams(ForkStreams **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 16) return cudaErrorInvalidDevice;
    ForkStreams &F = t_fork[dev];
    if (!F.ready) {
        e = cudaEventCreateWithFlags(&F.start, cudaEventDisableTiming);
        for (int i = 0; i < CMFW_MAX_MIXED_DESCS && e == cudaSuccess; ++i) {
            e = cudaStreamCreateWithFlags(&F.s[i], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&F.done[i], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) return e;
        F.ready = true;
    }
    *out = &F;
    return cudaSuccess;
}

// Per family, on its own stream forked from s and joined back into s: the
// singularity scan (persistent, cost-sorted queue) and the walk of its
// survivors only (tuning->prescan), or the walk of every trajectory. The
// sort comes first, on s (enqueue_mixed).
static cudaError_t enqueue_families_forked(const MixedArgs &M, const MixedLayout &L, int variant,
                                           const cmfw_mixed_tuning &tune, cudaStream_t s) {
    ForkStreams *F = nullptr;
    cudaError_t e = fork_streams(&F);
    if (e == cudaSuccess) e = cudaEventRecord(F->start, s);
    const bool prescan = tune.persistent && tune.prescan;
    int forked = 0;
    for (int f = 0; f < M.n_descs && e == cudaSuccess; ++f) {
        cudaStream_t fs = F->s[f];
        e = cudaStreamWaitEvent(fs, F->start, 0);
        if (e != cudaSuccess) break;
        forked = f + 1;
        e = enqueue_family_scan_walk(M, L, f, variant, tune, prescan, fs);
        const cudaError_t r = cudaEventRecord(F->done[f], fs);  // also after an error: the join needs it
        if (e == cudaSuccess) e = r;
    }
    // join every forked stream back, also after an error (a capture must
    // end with its branches joined)
    for (int f = 0; f < forked; ++f) {
        const cudaError_t j = cudaStreamWaitEvent(s, F->done[f], 0);
        if (e == cudaSuccess) e = j;
    }
    return e;
}

static cudaError_t enqueue_mixed(const MixedArgs &M, const MixedLayout &L, int variant,
                                 const cmfw_mixed_tuning &tune, cudaStream_t s) {
    const cudaError_t e = enqueue_sort(M, L, s);
    return e != cudaSuccess ? e : enqueue_families_forked(M, L, variant, tune, s);
}

}  // namespace cmfw

using namespace cmfw;

namespace {

cmfw_status cuda_fail(cudaError_t e, const char *what) {
    char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    return record_error(CMFW_ECUDA, msg);
}

cmfw_mixed_tuning default_tuning(int n_descs) {
    cmfw_mixed_tuning t;
    memset(&t, 0, sizeof(t));
    t.persistent = 1;
    t.prescan = 0;
    for (int i = 0; i < n_descs && i < CMFW_MAX_MIXED_DESCS; ++i) default_tile(t.tile[i]);
    return t;
}

// Candidate c of the autotuner's whole-batch stage: -2 the plain 256-thread
// grid everywhere (the fixed baseline), -1 the per-family choices, -3 the
// default tiles, -4 / -5 the default tiles / the per-family choices with the
// singularity prescan, 0..8 tile c (block blocks[c / 3], grab grabs[c % 3])
// for every family.
constexpr int kFirstCandidate = -5;
cmfw_mixed_tuning joint_candidate(const cmfw_mixed_tuning &per_family, int c, int n_descs, const int *blocks,
                                  const int *grabs) {
    cmfw_mixed_tuning t = per_family;
    if (c == -3 || c == -4) t = default_tuning(n_descs);
    if (c == -4 || c == -5) t.prescan = 1;
    if (c == -2) t.persistent = 0;
    if (c >= 0)
        for (int f = 0; f < n_descs; ++f) {
            t.tile[f].block_size = blocks[c / 3];
            t.tile[f].grab = grabs[c % 3];
            t.tile[f].ctas_per_sm = 0;
        }
    return t;
}

}  // namespace

struct cmfw_mixed_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void *owned_ws = nullptr;
};

extern "C" {

size_t cmfw_mixed_workspace_bytes(int n_traj, int n_descs) {
    if (n_traj < 0 || n_descs < 1 || n_descs > CMFW_MAX_MIXED_DESCS) return 0;
    return mixed_ws_bytes(n_traj, n_descs);
}

cmfw_status cmfw_walk_mixed(const cmfw_desc *descs, int n_descs, const cmfw_traj_in *d_in,
                            const cmfw_mixed_item *d_items, cmfw_traj_out *d_out, int n_traj, int h, int variant,
                            const cmfw_mixed_tuning *tuning, const cmfw_launch *launch, void *stream) {
    cmfw_status st = check_mixed(descs, n_descs, n_traj, h, variant);
    if (st != CMFW_OK || n_traj == 0) return st;
    if (!d_in || !d_items || !d_out) return record_error(CMFW_EINVAL, "NULL trajectory buffer");
    if (!launch || !launch->d_workspace || launch->workspace_bytes < mixed_ws_bytes(n_traj, n_descs))
        return record_error(CMFW_EINVAL, "a mixed batch needs a caller workspace of cmfw_mixed_workspace_bytes()");
    const MixedLayout L = mixed_layout(launch->d_workspace, n_traj);
    const MixedArgs M = make_args(descs, n_descs, d_in, d_items, d_out, n_traj, h, launch, L);
    const cmfw_mixed_tuning tune = tuning ? *tuning : default_tuning(n_descs);
    cudaError_t e = enqueue_mixed(M, L, variant, tune, (cudaStream_t)stream);
    return e == cudaSuccess ? CMFW_OK : cuda_fail(e, "mixed walk launch");
}

cmfw_status cmfw_mixed_autotune(const cmfw_desc *descs, int n_descs, const cmfw_traj_in *d_in,
                                const cmfw_mixed_item *d_items, cmfw_traj_out *d_out, int n_traj, int h,
                                int variant, const cmfw_launch *launch, int sample, cmfw_mixed_tuning *out,
                                void *stream) {
    if (!out) return record_error(CMFW_EINVAL, "NULL tuning output");
    cmfw_status st = check_mixed(descs, n_descs, n_traj, h, variant);
    if (st != CMFW_OK) return st;
    *out = default_tuning(n_descs);
    if (n_traj == 0) return CMFW_OK;
    if (!d_in || !d_items || !d_out) return record_error(CMFW_EINVAL, "NULL trajectory buffer");
    if (!launch || !launch->d_workspace || launch->workspace_bytes < mixed_ws_bytes(n_traj, n_descs))
        return record_error(CMFW_EINVAL, "a mixed batch needs a caller workspace of cmfw_mixed_workspace_bytes()");
    cudaStream_t s = (cudaStream_t)stream;
    const MixedLayout L = mixed_layout(launch->d_workspace, n_traj);
    MixedArgs M = make_args(descs, n_descs, d_in, d_items, d_out, n_traj, h, launch, L);
    cudaError_t e = enqueue_sort(M, L, s);
    std::vector<int> begin(n_descs + 1), order;
    if (e == cudaSuccess) e = cudaMemcpyAsync(begin.data(), L.begin, sizeof(int) * (n_descs + 1),
                                              cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "mixed autotune sort");
    order.resize(n_traj);
    e = cudaMemcpy(order.data(), L.order, sizeof(int) * (size_t)n_traj, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "mixed autotune order");
    if (sample <= 0) sample = 65536;
    // a strided sample of each family's sorted segment keeps its cost mix
    int *d_sorder = nullptr, *d_sbegin = nullptr, *d_snext = nullptr;
    e = cudaMalloc(&d_sorder, sizeof(int) * (size_t)sample);
    if (e == cudaSuccess) e = cudaMalloc(&d_sbegin, sizeof(int) * (CMFW_MAX_MIXED_DESCS + 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_snext, sizeof(int) * CMFW_MAX_MIXED_DESCS);
    cudaEvent_t a = nullptr, b = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    const int blocks[3] = {64, 128, 256};
    const int grabs[3] = {0, 32, 64};  // 0: plain grid, one trajectory per thread
    for (int f = 0; f < n_descs && e == cudaSuccess; ++f) {
        const int len = begin[f + 1] - begin[f];
        if (len <= 0) continue;
        const int m = len < sample ? len : sample;
        std::vector<int> so(m), sb(CMFW_MAX_MIXED_DESCS + 1, 0);
        for (int i = 0; i < m; ++i) so[i] = order[begin[f] + (int)(((long long)i * len) / m)];
        sb[f + 1] = m;
        for (int g = f + 2; g <= CMFW_MAX_MIXED_DESCS; ++g) sb[g] = m;
        e = cudaMemcpy(d_sorder, so.data(), sizeof(int) * m, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_sbegin, sb.data(), sizeof(int) * sb.size(), cudaMemcpyHostToDevice);
        MixedArgs Ms = M;
        Ms.order = d_sorder;
        Ms.begin = d_sbegin;
        Ms.next = d_snext;
        float best = 1e30f;
        for (int bi = 0; bi < 3 && e == cudaSuccess; ++bi)
            for (int gi = 0; gi < 3 && e == cudaSuccess; ++gi) {
                cmfw_mixed_tile tile;
                tile.block_size = blocks[bi];
                tile.grab = grabs[gi];
                tile.ctas_per_sm = 0;
                float ms = 0.f;
                for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // warm-up, then timed
                    e = cudaMemsetAsync(d_snext, 0, sizeof(int) * CMFW_MAX_MIXED_DESCS, s);
                    if (e == cudaSuccess) e = cudaEventRecord(a, s);
                    if (e == cudaSuccess) e = enqueue_family(Ms, f, variant, tile, 1, s);
                    if (e == cudaSuccess) e = cudaEventRecord(b, s);
                    if (e == cudaSuccess) e = cudaEventSynchronize(b);
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
                }
                if (e == cudaSuccess && ms < best) {
                    best = ms;
                    out->tile[f] = tile;
                }
            }
    }
    // The families walk side by side (enqueue_mixed), so the per-family
    // times do not add up: compare whole-batch tile sets on a joint sample
    // (every family's strided sample) -- the plain grid, the per-family
    // choices, and each tile for every family -- and keep the fastest.
    std::vector<int> so_all, sb_all(CMFW_MAX_MIXED_DESCS + 1, 0);
    for (int f = 0; f < n_descs; ++f) {
        const int len = begin[f + 1] - begin[f];
        const int m = len <= 0 ? 0 : (len < sample ? len : sample);
        for (int i = 0; i < m; ++i) so_all.push_back(order[begin[f] + (int)(((long long)i * len) / m)]);
        sb_all[f + 1] = (int)so_all.size();
    }
    for (int g = n_descs + 1; g <= CMFW_MAX_MIXED_DESCS; ++g) sb_all[g] = (int)so_all.size();
    int *d_jorder = nullptr;
    if (e == cudaSuccess && !so_all.empty()) {
        e = cudaMalloc(&d_jorder, sizeof(int) * so_all.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(d_jorder, so_all.data(), sizeof(int) * so_all.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_sbegin, sb_all.data(), sizeof(int) * sb_all.size(), cudaMemcpyHostToDevice);
        MixedArgs Mj = M;
        Mj.order = d_jorder;
        Mj.begin = d_sbegin;
        Mj.next = d_snext;
        const cmfw_mixed_tuning per_family = *out;
        std::vector<std::pair<float, int>> timed;  // (sample ms, candidate)
        for (int c = kFirstCandidate; c < 9 && e == cudaSuccess; ++c) {
            const cmfw_mixed_tuning t = joint_candidate(per_family, c, n_descs, blocks, grabs);
            float ms = 0.f;
            for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // warm-up, then timed
                e = cudaMemsetAsync(d_snext, 0, sizeof(int) * CMFW_MAX_MIXED_DESCS, s);
                if (e == cudaSuccess) e = cudaEventRecord(a, s);
                if (e == cudaSuccess) e = enqueue_families_forked(Mj, L, variant, t, s);
                if (e == cudaSuccess) e = cudaEventRecord(b, s);
                if (e == cudaSuccess) e = cudaEventSynchronize(b);
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
            }
            if (e == cudaSuccess) timed.push_back({ms, c});
        }
        // A sample ranks the candidates but can misjudge the whole batch's
        // tails: the fastest three on the sample, the default tiles (c = -3)
        // and the fixed baseline (the plain 256-thread grid, c = -2) are
        // timed on the whole batch, and the fastest of those is kept -- so
        // the tuning never loses to the default or the baseline by more than
        // the timing noise.
        std::sort(timed.begin(), timed.end());
        std::vector<int> finalists;
        for (size_t i = 0; i < timed.size() && finalists.size() < 3; ++i) finalists.push_back(timed[i].second);
        for (int must : {-2, -3})
            if (std::find(finalists.begin(), finalists.end(), must) == finalists.end()) finalists.push_back(must);
        float best = 1e30f;
        for (int c : finalists) {
            if (e != cudaSuccess) break;
            const cmfw_mixed_tuning t = joint_candidate(per_family, c, n_descs, blocks, grabs);
            // warm-up, then the better of two timed runs (the finalists are
            // often within a few per cent of each other)
            float ms = 1e30f;
            for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
                float m1 = 0.f;
                e = cudaEventRecord(a, s);
                if (e == cudaSuccess) e = enqueue_mixed(M, L, variant, t, s);
                if (e == cudaSuccess) e = cudaEventRecord(b, s);
                if (e == cudaSuccess) e = cudaEventSynchronize(b);
                if (e == cudaSuccess) e = cudaEventElapsedTime(&m1, a, b);
                if (rep > 0 && m1 < ms) ms = m1;
            }
            if (e == cudaSuccess && ms < best) {
                best = ms;
                *out = t;
            }
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(d_jorder);
    cudaFree(d_sorder);
    cudaFree(d_sbegin);
    cudaFree(d_snext);
    return e == cudaSuccess ? CMFW_OK : cuda_fail(e, "mixed autotune");
}

cmfw_status cmfw_mixed_graph_create(const cmfw_desc *descs, int n_descs, const cmfw_traj_in *d_in,
                                    const cmfw_mixed_item *d_items, cmfw_traj_out *d_out, int n_traj, int h,
                                    int variant, const cmfw_mixed_tuning *tuning, const cmfw_launch *launch,
                                    cmfw_mixed_graph **out) {
    if (!out) return record_error(CMFW_EINVAL, "NULL graph output");
    *out = nullptr;
    cmfw_status st = check_mixed(descs, n_descs, n_traj, h, variant);
    if (st != CMFW_OK) return st;
    if (n_traj > 0 && (!d_in || !d_items || !d_out)) return record_error(CMFW_EINVAL, "NULL trajectory buffer");
    cmfw_mixed_graph *g = new cmfw_mixed_graph();
    cmfw_launch L0 = {};
    if (launch) L0 = *launch;
    const size_t need = mixed_ws_bytes(n_traj, n_descs);
    if (!L0.d_workspace) {
        cudaError_t e = cudaMalloc(&g->owned_ws, need);
        if (e != cudaSuccess) {
            delete g;
            return record_error(CMFW_ENOMEM, "mixed graph workspace allocation failed");
        }
        L0.d_workspace = g->owned_ws;
        L0.workspace_bytes = need;
    } else if (L0.workspace_bytes < need) {
        delete g;
        return record_error(CMFW_EINVAL, "workspace below cmfw_mixed_workspace_bytes()");
    }
    const MixedLayout L = mixed_layout(L0.d_workspace, n_traj);
    const MixedArgs M = make_args(descs, n_descs, d_in, d_items, d_out, n_traj, h, &L0, L);
    const cmfw_mixed_tuning tune = tuning ? *tuning : default_tuning(n_descs);
    // occupancy queries and kernel lookups happen before the capture
    for (int f = 0; f < n_descs; ++f)
        if (!pick_mixed_variant(variant, descs[f])) {
            cmfw_mixed_graph_destroy(g);
            return record_error(CMFW_EUNSUPPORTED, "no kernel for a descriptor");
        }
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t e1 = n_traj > 0 ? enqueue_mixed(M, L, variant, tune, cs) : cudaSuccess;
        e = cudaStreamEndCapture(cs, &g->graph);
        if (e1 != cudaSuccess) e = e1;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (cs) cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        cmfw_mixed_graph_destroy(g);
        return cuda_fail(e, "mixed graph capture");
    }
    *out = g;
    return CMFW_OK;
}

cmfw_status cmfw_mixed_graph_launch(cmfw_mixed_graph *g, void *stream) {
    if (!g || !g->exec) return record_error(CMFW_EINVAL, "NULL graph");
    cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? CMFW_OK : cuda_fail(e, "mixed graph launch");
}

void cmfw_mixed_graph_destroy(cmfw_mixed_graph *g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->owned_ws) cudaFree(g->owned_ws);
    delete g;
}

}  // extern "C"
