// Chunked floating-point walk (default f64 / df64 path).
//
// A trajectory's walk is a product of N lattice-step matrices that depend
// only on the position, never on the accumulated product, so it can be cut
// into chunks walked independently and multiplied back together in order.
// Two kernels:
//
//  1. filter: one thread per trajectory runs the singularity tests of the
//     first S lattice steps (S = min(prefix_steps, N-2h-1)) without any
//     matrix work and keeps nothing but the verdict: a trajectory that
//     fails there is written invalid with its status, a survivor appends
//     its index to a list. Most trajectories that fail, fail here (zeta
//     starts hit a singular lead coefficient on their first y+ step). The
//     tests depend on the position only (FP64 column, denominators and
//     solve, which every arithmetic forms the same way), so the verdict is
//     the run arithmetic's; the survivors' first steps are walked again by
//     the chunk kernel's runs.
//  2. chunk: CTAs of 256 threads on a grid of one CTA per SM; each
//     survivor is walked by NP_b CTAs ("parts"), NP_b proportional to its
//     cost (axis steps per lattice step) so that all CTAs end together (at
//     most kMaxParts; with more survivors than CTAs, one CTA each). Steps
//     1..N form three segments [1, N-2h], [N-2h+1, N-h], [N-h+1, N] (the
//     snapshot depths are segment ends). Every segment's axis steps are
//     split evenly over its runs, one run per thread, so a run may start
//     and end inside a lattice step; each thread walks its run with the
//     same registers-only step as the sequential kernel (from rank 7 two
//     threads share a run, each holding half the rows), and a CTA
//     multiplies its runs of each segment in order by a shared-memory
//     tree. A trajectory walked in parts is finished by the part that
//     ends last: the parts publish their segment products to global
//     memory and count themselves in, and the last one to arrive (no CTA
//     ever waits for another) multiplies them in order, forms the three
//     snapshots seg0, seg0 * seg1, seg0 * seg1 * seg2 and reduces them.
//
// The latency of one trajectory drops from N L axis steps (L = sum |dir|)
// to about N L / (NP RT) axis steps (RT runs per CTA) + log2 RT + log2 NP
// matrix products; the total arithmetic is that of the sequential walk
// plus NP RT - 1 dense rank^3 products.
//
// Accuracy. Multiplying runs together is a different association of the
// same matrix product. A run started from the identity can pass through
// directions that the true walk state never excites (early in a walk, while
// the positions are still small, the product can grow transiently along
// them); rounding at that size, once multiplied into the true state, is
// amplified. The f64 variant therefore walks its runs and multiplies them in
// double-double (ArithDD, about 106 bits, on the FP64 pipe): rounding inside
// the runs and the tree then sits far below what the sequential f64 walk
// commits, and the results keep the sequential walk's accuracy. The
// per-step matrices themselves (column, 1/a) are formed in FP64 exactly as
// in the sequential walk. CMFW_F_PLAIN_RUNS selects plain-FP64 runs (fewer
// instructions, no such guarantee); df64 runs in float-float with FP64
// products (ArithFF).
#include <algorithm>
#include <mutex>
#include <vector>

#include "walk_arith.cuh"

namespace cmfw {

struct ChunkArgs {
    WalkArgs w;
    int *list;                        // n_traj survivor indices
    int *count;                       // survivors
    int *cost;                        // n_traj: axis steps per lattice step of each listed survivor
    int *arrive;                      // nslots: parts finished, per survivor walked in parts
    void *parts;                      // nslots x 3 segment products of the parts (combine arithmetic)
    int *parts_e;                     // nslots x 3 their exponents
    unsigned long long *parts_fail;   // nslots earliest failure keys
    int nslots;
    // CTAs that survivors walked in parts are shared out over: one per SM,
    // whatever the kernel's occupancy, and at most 32 * kLaneItems
    int part_budget;
    int prefix_steps;
};

// Threads per CTA of the filter kernel: 64, so that a batch of 10^4
// trajectories spreads over every SM.
constexpr int kFilterThreads = 64;

template <int P_, int Q_, int DIM>
__global__ void __launch_bounds__(kFilterThreads) walk_prefix_kernel(ChunkArgs C) {
    // the chunk kernel may be scheduled now: it waits for this grid's end
    // (cudaGridDependencySynchronize) before it reads anything written here
    cudaTriggerProgrammaticLaunchCompletion();
    const WalkArgs &W = C.w;
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= W.n_traj) return;
    const int P = (P_ > 0) ? P_ : W.p;
    const int Q = (P_ > 0) ? Q_ : W.q;
    const int naxes = P + Q;
    const cmfw_traj_in &in = W.in[t];
    int absd[NAX];
    uint32_t neg;
    const int maxabs = load_direction<NAX>(in, naxes, absd, neg);
    if (maxabs < 0) { write_invalid(W, t, CMFW_TRAJ_STEP_CAP); return; }
    if (W.N <= 0 || W.h <= 0 || W.N - 2 * W.h <= 0) { write_invalid(W, t, CMFW_TRAJ_BAD_DEPTH); return; }
    double pos[NAX];
#pragma unroll
    for (int a = 0; a < NAX; ++a) pos[a] = (a < naxes) ? in.start[a] : 0.0;
    const StepConst K = make_step_const(P, Q, DIM, W.z);
    // The singularity tests alone: a step that would leave the walk matrix
    // non-finite without failing a test is found by the chunk kernel at the
    // same lattice step (its runs test the matrix at every lattice-step end)
    const int S = min(C.prefix_steps, W.N - 2 * W.h - 1);
    for (int step = 1; step <= S; ++step) {
        const int st = lattice_step_tests<DIM, NAX, PM, QM>(pos, absd, neg, maxabs, K);
        if (st != CMFW_TRAJ_OK) { write_invalid(W, t, st); return; }
    }
    const int at = atomicAdd(C.count, 1);
    C.list[at] = t;
    int L = 0;
#pragma unroll
    for (int a = 0; a < NAX; ++a) L += absd[a];
    C.cost[at] = L;
}

// Threads per CTA of the chunk kernel, and threads per run: up to rank 6 a
// thread holds a run's whole walk state (25 or 36 double-double entries);
// from rank 7 two adjacent threads share a run, each with half the rows
// (the rows of a walk evolve independently), since 49 or 64 double-double
// entries would not fit one thread's registers. Runs, and shared product
// slots, per CTA = threads / threads per run.
__host__ __device__ constexpr int chunk_threads(int dim) { return 256; }
__host__ __device__ constexpr int chunk_pair(int dim) { return dim >= 7 ? 2 : 1; }
__host__ __device__ constexpr int chunk_runs(int dim) { return chunk_threads(dim) / chunk_pair(dim); }

// CTA-cooperative products: every task multiplies two DIM x DIM matrices
// (matrix-exponent form) in the combine arithmetic, one result entry per
// work item spread over the NT threads (ILP independent entries in flight
// per thread); the entries go to a staging area first, so a task may write
// over its first operand, and each result is rescaled by a power of two so
// that its largest entry lies in [1, 2) (per-task maximum through a shared
// atomic).
template <class CA>
struct ProdTask {
    const typename CA::T *a, *b;
    typename CA::T *c;
    int ea, eb;
    int *ec;
};

template <int DIM, class CA, int NT>
__device__ __forceinline__ void par_products(const ProdTask<CA> *tasks, int ntasks, int *pmax,
                                             typename CA::T *stage) {
    typedef typename CA::T CT;
    constexpr int DD = DIM * DIM;
    constexpr int ILP = 4;
    const int nw = ntasks * DD;
#pragma unroll 1
    for (int w0 = threadIdx.x; w0 < nw; w0 += ILP * NT) {
        CT x[ILP];
#pragma unroll
        for (int u = 0; u < ILP; ++u) {
            const int w = w0 + u * NT;
            if (w < nw) {
                const ProdTask<CA> &T = tasks[w / DD];
                const int e = w % DD, i = e / DIM, j = e % DIM;
                x[u] = CA::template dot<DIM>(T.a + i * DIM, 1, T.b + j, DIM);
            }
        }
#pragma unroll
        for (int u = 0; u < ILP; ++u) {
            const int w = w0 + u * NT;
            if (w < nw) {
                stage[w] = x[u];
                atomicMax(&pmax[w / DD], CA::hexp(x[u]));
            }
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int w = threadIdx.x; w < nw; w += NT) {
        const ProdTask<CA> &T = tasks[w / DD];
        const int hm = pmax[w / DD];
        const int be = (hm != 0 && hm < 0x7ff00000) ? (hm >> 20) - 1023 : 0;
        T.c[w % DD] = CA::scale(stage[w], be);
        if (w % DD == 0) *T.ec = T.ea + T.eb + be;
    }
    __syncthreads();
}

// Dynamic shared memory of the chunk kernel: RT run products + 3 snapshot
// matrices (RT = runs per CTA), their exponents, RT/2 product tasks with
// their maxima, and one region that holds the threads' positions during
// the runs and the products' staging area afterwards. (Static: the
// threads' run ends and the per-launch geometry, about 2.4 KB; rank 6 in
// double-double, the largest user, stays below the 227 KB a CTA may hold.)
template <class CT>
__host__ __device__ constexpr size_t chunk_union_bytes(int dim) {
    return (size_t)CMFW_MAX_AXES * chunk_threads(dim) * sizeof(double) >
                   (size_t)(chunk_runs(dim) / 2) * dim * dim * sizeof(CT)
               ? (size_t)CMFW_MAX_AXES * chunk_threads(dim) * sizeof(double)
               : (size_t)(chunk_runs(dim) / 2) * dim * dim * sizeof(CT);
}
template <class CT>
__host__ __device__ constexpr size_t chunk_union_offset(int dim) {
    return ((size_t)(chunk_runs(dim) + 3) * dim * dim * sizeof(CT) + (chunk_runs(dim) + 3) * sizeof(int) + 15) /
               16 * 16 +
           (size_t)(chunk_runs(dim) / 2) * (sizeof(ProdTask<ArithF64>) + sizeof(int));
}
template <class CT>
__host__ __device__ constexpr size_t chunk_smem_bytes(int dim) {
    return (chunk_union_offset<CT>(dim) + 15) / 16 * 16 + chunk_union_bytes<CT>(dim);
}

// In-order products of up to three groups of consecutive shared-memory
// matrices (matrix-exponent form): group k holds slots gbase[k] ..
// gbase[k] + gcnt[k] - 1 and ends with its product in slot gbase[k]. One
// tree level at a time: at stride st the products are slot a = gbase[k] +
// 2 st m times slot a + st (for a + st inside the group), enumerated in
// closed form. Every product's entries take whole warps (DD entries padded
// to EW = 32 or 64 lanes), each thread ILP entries in flight; a warp's
// largest exponent is one reduction. Up to rank 5 (one warp per product)
// each warp writes its product back rescaled at once: one barrier a level.
// Above, the entries are staged and written back once both warps' maxima
// are in: two barriers a level. No atomics. wmax holds 2 ints per product.
// (Out of line: its registers are then not counted against the walk
// state's.)
__device__ __forceinline__ int level_tasks(int cnt, int st) { return cnt > st ? (cnt - st - 1) / (2 * st) + 1 : 0; }

template <int DIM, class CA, int NT>
__device__ __noinline__ void group_products(typename CA::T *slots, int *sexp, const int *gbase, const int *gcnt,
                                            int *wmax, typename CA::T *stage) {
    typedef typename CA::T CT;
    constexpr int DD = DIM * DIM;
    constexpr int EW = 32 * ((DD + 31) / 32);  // lanes per product
    constexpr int ILP = 4;
    const int tid = threadIdx.x, lane = tid & 31;
    const int g0 = gbase[0], g1 = gbase[1], g2 = gbase[2];
    const int c0 = gcnt[0], c1 = gcnt[1], c2 = gcnt[2];
    const int cmax = max(c0, max(c1, c2));
    for (int st = 1; st < cmax; st <<= 1) {
        const int n0 = level_tasks(c0, st), n1 = level_tasks(c1, st), n2 = level_tasks(c2, st);
        const int nt = n0 + n1 + n2;
        const int nw = nt * EW;
#pragma unroll 1
        for (int w0 = tid; w0 < nw; w0 += ILP * NT) {
            CT x[ILP];
#pragma unroll
            for (int u = 0; u < ILP; ++u) {
                const int w = w0 + u * NT;  // warp-uniform: nw is a multiple of 32
                const int tau = w / EW, e = w % EW;
                if (w < nw && e < DD) {
                    const int i = e / DIM, j = e % DIM;
                    const int a = tau < n0 ? g0 + 2 * st * tau
                                           : (tau < n0 + n1 ? g1 + 2 * st * (tau - n0) : g2 + 2 * st * (tau - n0 - n1));
                    const CT *A = slots + a * DD, *B = slots + (a + st) * DD;
                    x[u] = CA::template dot<DIM>(A + i * DIM, 1, B + j, DIM);
                }
            }
#pragma unroll
            for (int u = 0; u < ILP; ++u) {
                const int w = w0 + u * NT;
                if (w < nw) {
                    const int tau = w / EW, e = w % EW;
                    const unsigned hx = e < DD ? (unsigned)CA::hexp(x[u]) : 0u;
                    const unsigned hm = __reduce_max_sync(0xffffffffu, hx);
                    if constexpr (EW == 32) {
                        // one warp holds the whole product: every lane has
                        // read its operands before the reduction, and no
                        // other product of this level reads slot a, so the
                        // result goes straight back into slot a
                        const int a = tau < n0 ? g0 + 2 * st * tau
                                               : (tau < n0 + n1 ? g1 + 2 * st * (tau - n0)
                                                                : g2 + 2 * st * (tau - n0 - n1));
                        const int be = (hm != 0 && hm < 0x7ff00000u) ? (int)(hm >> 20) - 1023 : 0;
                        if (e < DD) slots[a * DD + e] = CA::scale(x[u], be);
                        if (e == 0) sexp[a] = sexp[a] + sexp[a + st] + be;
                    } else {
                        if (lane == 0) wmax[2 * tau + e / 32] = (int)hm;
                        if (e < DD) stage[tau * DD + e] = x[u];
                    }
                }
            }
        }
        __syncthreads();
        if constexpr (EW > 32) {
#pragma unroll 1
            for (int w = tid; w < nt * DD; w += NT) {
                const int tau = w / DD, e = w % DD;
                const int a = tau < n0 ? g0 + 2 * st * tau
                                       : (tau < n0 + n1 ? g1 + 2 * st * (tau - n0) : g2 + 2 * st * (tau - n0 - n1));
                const int hm = max(wmax[2 * tau], wmax[2 * tau + 1]);
                const int be = (hm != 0 && hm < 0x7ff00000) ? (hm >> 20) - 1023 : 0;
                slots[a * DD + e] = CA::scale(stage[w], be);
                if (e == 0) sexp[a] = sexp[a] + sexp[a + st] + be;
            }
            __syncthreads();
        }
    }
}

// Failure key of axis step a (0-based over the whole walk): the earliest
// failing step of a trajectory is the smallest key.
__device__ __forceinline__ unsigned long long fail_key(long long a, int status) {
    return ((unsigned long long)a << 4) | (unsigned)status;
}
constexpr unsigned long long kNoFailure = ~0ull;

// Lanes of the thread pair that shares a run (G = 2), for shuffles.
__device__ __forceinline__ unsigned pair_mask() { return 3u << ((threadIdx.x & 31) & ~1u); }

// Walks axis steps [alo, *ahi) of a trajectory into the R rows m that this
// thread holds (G threads share a run, each with its own rows and the same
// position sequence). Axis step a is step a % L (in the plan's order) of
// lattice step a / L + 1, L the plan's axis steps per lattice step; pos
// holds the position at the start of lattice step alo / L + 1. Failures go
// to *fail as fail_key; at each lattice-step end the walk stops early if a
// smaller key is there. The non-finite test of the sequential walk runs at
// every lattice-step end inside the run and at the run's end, over the rows
// of all G threads. The threads of a run take every branch together (the
// step tests depend on the position only, and the decisions at
// lattice-step ends are combined), so their shuffles always pair up. (The
// run's end is read from shared memory, which keeps it out of the
// registers the walk state needs.)
template <int DIM, int NAX, int PM, int QM, class A, int NT, int R, int G>
__device__ __forceinline__ void walk_axis_range(typename A::T (&m)[R][DIM], int (&ex)[R], const SmemPos<NT> &pos,
                                                const LevelPlan &L, const StepConst &K, long long alo,
                                                const long long *ahi, unsigned long long *fail) {
    if (alo >= *ahi) return;
    volatile unsigned long long *vf = fail;
    int skip = (int)(alo % L.L);  // axis steps of the first lattice step before the run
    long long a = alo - skip;
    while (true) {
        for (int i = 0; i < L.k; ++i) {
            const uint32_t lm = L.mask[i];
            const int lo = L.thr[i + 1];
            for (int level = L.thr[i]; level > lo; --level) {
                uint32_t mask = lm;
                while (mask) {
                    const int axis = top_axis(mask);
                    mask &= ~(1u << axis);
                    const bool up = (L.up >> axis) & 1u;
                    if (a >= *ahi) goto run_end;
                    if (skip > 0) {
                        pos_move<NAX>(pos, axis, up ? 1.0 : -1.0);
                        --skip;
                    } else {
                        const int st = axis_step<DIM, NAX, PM, QM, A>(m, ex, pos, axis, up, K);
                        if (st != CMFW_TRAJ_OK) {
                            atomicMin(fail, fail_key(a, st));
                            return;
                        }
                    }
                    ++a;
                }
            }
        }
        {
            // (an identity, before the run's first step, is healthy)
            int bits = health_bits<A, R, DIM>(m) | (*vf < fail_key(a, 0) ? 4 : 0);
            if (G == 2) bits |= __shfl_xor_sync(pair_mask(), bits, 1);
            if (!(bits & 1) || (bits & 2)) {
                atomicMin(fail, fail_key(a - 1, CMFW_TRAJ_NONFINITE));
                return;
            }
            if (a >= *ahi || (bits & 4)) return;  // run done, or an earlier axis step failed
        }
    }
run_end:
    int bits = health_bits<A, R, DIM>(m);
    if (G == 2) bits |= __shfl_xor_sync(pair_mask(), bits, 1);
    if (!(bits & 1) || (bits & 2)) atomicMin(fail, fail_key(a - 1, CMFW_TRAJ_NONFINITE));
}

// A run's rows (row r * G + h of the walk in this thread's row r) in
// matrix-exponent form: the largest row exponent among non-zero rows of
// the G threads becomes the matrix exponent (returned), rows more than
// 2^1000 below it flush to zero, and each thread writes its rows to out.
template <int DIM, int R, int G, class A>
__device__ __forceinline__ int rows_to_matrix_exponent(const typename A::T (&m)[R][DIM], const int (&ex)[R], int h,
                                                       typename A::Combine::T *out /* DIM*DIM */) {
    typedef typename A::Combine C;
    int emax = -0x40000000;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        bool nz = false;
#pragma unroll
        for (int j = 0; j < DIM; ++j) nz |= A::nonzero(m[r][j]);
        if (nz && r * G + h < DIM) emax = max(emax, ex[r]);
    }
    if (G == 2) emax = max(emax, __shfl_xor_sync(pair_mask(), emax, 1));
    if (emax == -0x40000000) emax = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int rg = r * G + h;
        if (rg < DIM) {
            const int be = max(emax - ex[r], 0);
            const bool keep = be < 1000;
#pragma unroll
            for (int j = 0; j < DIM; ++j) {
                typename C::T v = A::to_combine(m[r][j]);
                out[rg * DIM + j] = keep ? C::scale(v, be) : C::from(0.0);
            }
        }
    }
    return emax;
}

// The run geometry of a trajectory walked by np parts of rt runs each:
// blocks of x lattice steps cut into c pieces (see walk_chunk_kernel),
// with each segment's first block and first run.
__device__ __forceinline__ void run_geometry(int N, int h, int np, int rt, int g, int *c_out, int *x_out,
                                          int *blockbase, int *segbase, int *segT) {
    const int n[3] = {N - 2 * h, h, h};
    int best_c = 1, best_x = 1 << 30;
    for (int c = 1; c <= 8 && (rt / c) * g >= 32; c <<= 1) {
        const int cap = np * (rt / c);
        int x = max(1, (N + cap - 1) / cap);
        while ((n[0] + x - 1) / x + (n[1] + x - 1) / x + (n[2] + x - 1) / x > cap) ++x;
        if ((long long)x * best_c < (long long)best_x * c) {
            best_c = c;
            best_x = x;
        }
    }
    *c_out = best_c;
    *x_out = best_x;
    int bb = 0;
    for (int k = 0; k < 3; ++k) {
        const int nb = (n[k] + best_x - 1) / best_x;
        blockbase[k] = bb;
        segbase[k] = bb * best_c;
        segT[k] = nb * best_c;
        bb += nb;
    }
}

// CTAs that walk one trajectory together, at most, and the survivors per
// lane of the warp that shares out the parts: the host caps the part budget
// at 32 x kLaneItems, so the warp sees every survivor of a balanced batch.
constexpr int kMaxParts = 16;
constexpr int kLaneItems = 10;
constexpr int kMaxPartBudget = 32 * kLaneItems;

__device__ __forceinline__ double ldcg_d(const double *p) { return __ldcg(p); }
__device__ __forceinline__ dd ldcg_d(const dd *p) { return dd{__ldcg(&p->hi), __ldcg(&p->lo)}; }

template <int P_, int Q_, int DIM, class A>
__global__ void __launch_bounds__(chunk_threads(DIM), 1) walk_chunk_kernel(ChunkArgs C) {
    constexpr int NT = chunk_threads(DIM);
    constexpr int G = chunk_pair(DIM);   // threads per run
    constexpr int RT = NT / G;           // runs (product slots) per CTA
    constexpr int R = (DIM + G - 1) / G; // walk rows per thread
    typedef typename A::T T;
    typedef typename A::Combine CA;
    typedef typename CA::T CT;
    const WalkArgs &W = C.w;
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    constexpr int DD = DIM * DIM;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CT *smem = (CT *)smem_raw;                  // RT run products + 3 snapshot matrices
    int *sexp = (int *)(smem + (RT + 3) * DD);  // RT + 3 exponents
    ProdTask<CA> *tasks = (ProdTask<CA> *)(((uintptr_t)(sexp + RT + 3) + 15) & ~(uintptr_t)15);  // RT / 2
    int *pmax = (int *)(tasks + RT / 2);        // RT / 2
    unsigned char *ureg = smem_raw + (chunk_union_offset<CT>(DIM) + 15) / 16 * 16;
    double *s_pos = (double *)ureg;             // during the runs: [NAX][NT] positions
    CT *stage = (CT *)ureg;                     // afterwards: product staging
    __shared__ int s_ok, s_last;
    // snapshot reduction: largest |entry| bits and a non-zero flag per
    // snapshot, and the limit selection
    __shared__ unsigned long long s_g[3];
    __shared__ int s_nz[3], s_kany, s_kait, s_npush, s_nbefore;
    __shared__ double s_ls[3];
    // earliest failing axis step of this CTA's runs (fail_key), and of the
    // trajectory once the parts are combined
    __shared__ unsigned long long s_fail, s_fkey;
    __shared__ LevelPlan s_plan;
    // groups of shared-memory products for group_products
    __shared__ int s_gbase[3], s_gcnt[3];
    __shared__ StepConst s_K;
    __shared__ long long s_ahi[NT];  // each thread's run end
    __shared__ int s_t;  // the trajectory walked
    const int tid = threadIdx.x;
    const int P = (P_ > 0) ? P_ : W.p;
    const int Q = (P_ > 0) ? Q_ : W.q;
    const int naxes = P + Q;
    if (tid == 0) s_K = make_step_const(P, Q, DIM, W.z);

    // Parts per trajectory. With no more survivors than the part budget B
    // (one CTA per SM), every survivor b gets NP_b = min(kMaxParts,
    // ceil(w_b / t)) CTAs, w_b = its axis steps per lattice step (its
    // walk's cost), t the smallest work per CTA (in sixteenths) whose parts
    // fit B: long walks get more CTAs, so the CTAs end at about the same
    // time. Survivors take consecutive CTAs in list order; a CTA walks one
    // part and is done (CTAs past the parts exit). With more survivors than
    // B, every survivor is one CTA's and the CTAs stride over the list.
    // B is fixed by the SM count alone, not by how many CTAs of this build
    // fit an SM: NP_b, hence the run geometry and the association of the
    // product (and so every rounding), depend on the batch and the device
    // only. Warp 0 finds this CTA's part; the values are kept in shared
    // memory, like the run geometry below.
    __shared__ int s_count, s_bal, s_b0, s_part0, s_np0, s_first0;
    // The filter kernel is launched before this one with programmatic
    // stream serialisation: wait (in hardware) until it has finished and
    // its survivor list is visible. Nothing above reads its outputs.
    cudaGridDependencySynchronize();
    if (tid < 32) {
        const int count = *C.count;
        const int Gr = min(min((int)gridDim.x, C.nslots), min(C.part_budget, kMaxPartBudget));
        // CMFW_F_BATCH_INVARIANT: one CTA per survivor whatever the batch, so
        // a trajectory's run geometry (and every rounding) is the same in
        // every batch
        const bool bal = count > 0 && count <= Gr && !(W.flags & CMFW_F_BATCH_INVARIANT);
        int b0 = -1, part0 = 0, np0 = 1, first0 = 0;
        if (bal) {
            int w[kLaneItems];
            int wmax = 1;
#pragma unroll
            for (int q = 0; q < kLaneItems; ++q) {
                const int b = tid + 32 * q;
                w[q] = b < count ? 16 * max(1, C.cost[b]) : 0;
                wmax = max(wmax, w[q]);
            }
            wmax = (int)__reduce_max_sync(0xffffffffu, (unsigned)wmax);
            int lo = 1, hi = wmax;  // at hi every survivor has one part
            while (lo < hi) {
                const int mid = (lo + hi) / 2;
                int parts = 0;
#pragma unroll
                for (int q = 0; q < kLaneItems; ++q)
                    if (w[q] > 0) parts += min(kMaxParts, (w[q] + mid - 1) / mid);
                parts = (int)__reduce_add_sync(0xffffffffu, (unsigned)parts);
                if (parts <= Gr) hi = mid; else lo = mid + 1;
            }
            if (tid == 0) {
                int at = 0;
                for (int b = 0; b < count; ++b) {
                    const int np = min(kMaxParts, (16 * max(1, C.cost[b]) + lo - 1) / lo);
                    if ((int)blockIdx.x < at + np) {
                        b0 = b;
                        part0 = blockIdx.x - at;
                        np0 = np;
                        first0 = at;
                        break;
                    }
                    at += np;
                }
            }
        }
        if (tid == 0) {
            s_count = count;
            s_bal = bal;
            s_b0 = b0;
            s_part0 = part0;
            s_np0 = np0;
            s_first0 = first0;
        }
    }
    __syncthreads();

    // The walk's three segments of lattice steps [1, N-2h], [N-2h+1, N-h],
    // [N-h+1, N] (their ends are the snapshot depths) are tiled by blocks of
    // x lattice steps (a segment's last block may be shorter), and every
    // block is cut into c pieces at the same axis-step offsets: piece i of a
    // block covers axis steps floor(i x L / c) .. floor((i+1) x L / c) of it
    // (L = sum |dir|). One piece is one thread's run. Piece i of every block
    // goes to warps of its own, so the threads of a warp start their runs at
    // the same offset inside a lattice step and walk the same number of axis
    // steps: no divergence. Runs are numbered block by block (run j = piece
    // j % c of block j / c), part p holds runs [p RT, (p+1) RT) and puts run
    // j's product in shared slot j - p RT, so a segment's runs sit in
    // consecutive slots in walk order. (c, x) minimise the run length x / c
    // over the blocks the trajectory's NP parts can hold. Kept in shared
    // memory and re-derived where needed, so that none of it holds a
    // register across the runs.
    __shared__ int s_c, s_x, s_blockbase[3], s_segbase[3], s_segT[3];
    // the part this CTA walks: trajectory list index, part, parts, and the
    // product slot of part 0
    __shared__ int s_ub, s_upart, s_unp, s_ufirst;

    for (int round = 0;; ++round) {
        if (tid == 0) {
            if (s_bal) {
                s_ub = round == 0 ? s_b0 : -1;
                s_upart = s_part0;
                s_unp = s_np0;
                s_ufirst = s_first0;
            } else {
                const int b = blockIdx.x + round * gridDim.x;
                s_ub = b < s_count ? b : -1;
                s_upart = 0;
                s_unp = 1;
                s_ufirst = 0;
            }
            if (s_ub >= 0) {
                const int t = C.list[s_ub];
                s_t = t;
                s_fail = kNoFailure;
                int absd[NAX];
                uint32_t neg;
                const int maxabs = load_direction<NAX>(W.in[t], naxes, absd, neg);
                make_level_plan<NAX>(absd, neg, maxabs, s_plan);
                run_geometry(W.N, W.h, s_unp, RT, G, &s_c, &s_x, s_blockbase, s_segbase, s_segT);
            }
        }
        __syncthreads();
        if (s_ub < 0) break;  // uniform over the CTA
        // this thread's rows of the walk (row r * G + h in row r; a row past
        // DIM, in the second thread of a pair at odd rank, stays zero)
        T m[R][DIM];
        int ex[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            ex[r] = 0;
#pragma unroll
            for (int j = 0; j < DIM; ++j) m[r][j] = A::from((r * G + tid % G == j) ? 1.0 : 0.0);
        }
        {
            // this thread's run: piece i of block B
            const int NB = RT / s_c, v = tid / G;
            const int B = s_upart * NB + v % NB, i = v / NB;
            const int k = B < s_blockbase[1] ? 0 : (B < s_blockbase[2] ? 1 : 2);
            const int nk = k == 0 ? W.N - 2 * W.h : W.h;
            const int first = k == 0 ? 1 : (k == 1 ? W.N - 2 * W.h + 1 : W.N - W.h + 1);
            const int sb = first + (B - s_blockbase[k]) * s_x;  // the block's first lattice step
            const int se = min(sb + s_x, first + nk);            // one past its last
            const long long Lk = s_plan.L;
            const long long b0 = (long long)(sb - 1) * Lk;
            long long alo = b0 + (long long)i * s_x * Lk / s_c;
            long long ahi = min(b0 + (long long)(i + 1) * s_x * Lk / s_c, (long long)(se - 1) * Lk);
            if (sb >= first + nk) alo = ahi = 0;  // beyond the last block: no run
            s_ahi[tid] = ahi;
            const cmfw_traj_in &in = W.in[s_t];
            const SmemPos<NT> pos{s_pos + tid};
            // lattice steps completed before the run (a zero direction has
            // no axis steps: every run is empty)
            const double s0 = Lk > 0 ? (double)(alo / Lk) : 0.0;
#pragma unroll
            for (int a = 0; a < NAX; ++a) {
                const double d = (a < naxes) ? (double)in.dir[a] : 0.0;
                pos.p[a * NT] = (a < naxes) ? in.start[a] + s0 * d : 0.0;
            }
            walk_axis_range<DIM, NAX, PM, QM, A, NT, R, G>(m, ex, pos, s_plan, s_K, alo, s_ahi + tid, &s_fail);
        }
        {
            const int NB = RT / s_c, v = tid / G;
            const int slot = (v % NB) * s_c + v / NB;
            const int e = rows_to_matrix_exponent<DIM, R, G, A>(m, ex, tid % G, smem + slot * DD);
            if (tid % G == 0) sexp[slot] = e;
        }
        const int b = s_ub, part = s_upart;
        if (tid == 0) {
            // this CTA's share of each segment's runs, in shared slots
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int b0 = max(s_segbase[k], part * RT);
                const int b1 = min(s_segbase[k] + s_segT[k], (part + 1) * RT);
                s_gbase[k] = b0 - part * RT;
                s_gcnt[k] = max(0, b1 - b0);
            }
        }
        __syncthreads();
        // in-order tree product of this CTA's runs of each segment
        group_products<DIM, CA, NT>(smem, sexp, s_gbase, s_gcnt, (int *)tasks, stage);

        const int NP = s_unp;
        if (NP > 1) {
            // publish this part's segment products; the last part to
            // finish combines them (no CTA waits for another)
            const size_t slot = (size_t)s_ufirst + part;
            CT *pp = (CT *)C.parts + slot * 3 * DD;
            for (int i = tid; i < 3 * DD; i += NT) {
                const int k = i / DD;
                if (s_gcnt[k] > 0) pp[i] = smem[s_gbase[k] * DD + i % DD];
            }
            if (tid < 3 && s_gcnt[tid] > 0) C.parts_e[slot * 3 + tid] = sexp[s_gbase[tid]];
            if (tid == 0) C.parts_fail[slot] = s_fail;
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = atomicAdd(&C.arrive[b], 1) == NP - 1;
            __syncthreads();
            if (!s_last) break;  // uniform over the CTA; a part is a CTA's only work
            __threadfence();
            if (tid == 0) {
                unsigned long long fk = kNoFailure;
                for (int q = 0; q < NP; ++q) fk = min(fk, __ldcg(&C.parts_fail[(size_t)s_ufirst + q]));
                s_fkey = fk;
                // segment k's products are those of parts q0 .. q1, in order
                int at = 0;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int q0 = s_segbase[k] / RT, q1 = (s_segbase[k] + s_segT[k] - 1) / RT;
                    s_gbase[k] = at;
                    s_gcnt[k] = q1 - q0 + 1;
                    at += q1 - q0 + 1;
                }
            }
            __syncthreads();
            if (s_fkey == kNoFailure) {
                const int nslot = s_gbase[2] + s_gcnt[2];
                for (int i = tid; i < nslot * DD; i += NT) {
                    const int sl = i / DD;
                    const int k = sl < s_gbase[1] ? 0 : (sl < s_gbase[2] ? 1 : 2);
                    const int q = s_segbase[k] / RT + (sl - s_gbase[k]);
                    const size_t src = ((size_t)s_ufirst + q) * 3 + k;
                    smem[i] = ldcg_d((const CT *)C.parts + src * DD + i % DD);
                    if (i % DD == 0) sexp[sl] = __ldcg(&C.parts_e[src]);
                }
                __syncthreads();
                group_products<DIM, CA, NT>(smem, sexp, s_gbase, s_gcnt, (int *)tasks, stage);
            }
        } else {
            if (tid == 0) s_fkey = s_fail;
            __syncthreads();
        }

        // the combined trajectory: segment products in slots s_gbase[k]
        const int t = s_t;
        CT *x = smem + RT * DD;
        int *xe = sexp + RT;
        if (s_fkey != kNoFailure) {
            if (tid == 0) write_invalid(W, t, (int)(s_fkey & 15));
        } else {
            // snapshots: seg0, then * seg1, then * seg2
            for (int i = tid; i < DD; i += NT) x[i] = smem[s_gbase[0] * DD + i];
            if (tid == 0) {
                xe[0] = sexp[s_gbase[0]];
                s_ok = 1;
            }
            __syncthreads();
            for (int k = 1; k < 3; ++k) {
                if (tid == 0) {
                    tasks[0] = ProdTask<CA>{x + (k - 1) * DD, smem + s_gbase[k] * DD, x + k * DD, xe[k - 1],
                                            sexp[s_gbase[k]], &xe[k]};
                    pmax[0] = 0;
                }
                __syncthreads();
                par_products<DIM, CA, NT>(tasks, 1, pmax, stage);
            }
            // the snapshots in the reference's form, in shared memory (the
            // staging area is free once the products are done). The rows of
            // a snapshot share its exponent xe[k], so the reference's
            // normalisation (normalise_rows) is a division by the largest
            // |entry| g_k and log_scale_k = xe[k] ln 2 + log g_k; the largest
            // entry is gathered on the bit patterns (non-negative doubles
            // order like their bits).
            double *snap = (double *)stage;
            int *snap_e = (int *)(snap + 3 * DD);
            if (tid < 3) {
                s_g[tid] = 0ull;
                s_nz[tid] = 0;
            }
            __syncthreads();
            for (int i = tid; i < 3 * DD; i += NT) {
                const double v = CA::to(x[i]);
                snap[i] = v;
                if (!isfinite(v)) {
                    atomicAnd(&s_ok, 0);
                } else if (v != 0.0) {
                    s_nz[i / DD] = 1;
                    atomicMax(&s_g[i / DD], (unsigned long long)__double_as_longlong(fabs(v)));
                }
            }
            if (tid < 3 * DIM) snap_e[tid] = xe[tid / DIM];
            __syncthreads();
            if (tid == 0 && !(s_nz[0] && s_nz[1] && s_nz[2])) s_ok = 0;  // a zero snapshot
            __syncthreads();
            if (!s_ok) {
                if (tid == 0) write_invalid(W, t, CMFW_TRAJ_NONFINITE);
            } else {
                for (int i = tid; i < 3 * DD; i += NT) snap[i] *= 1.0 / __longlong_as_double((long long)s_g[i / DD]);
                if (tid < 3) s_ls[tid] = (0.0 + (double)xe[tid] * CMFW_LN2) + log(__longlong_as_double((long long)s_g[tid]));
                if (tid == 0) {
                    s_kany = 0x7fffffff;
                    s_kait = 0x7fffffff;
                    s_npush = 0;
                    s_nbefore = 0;
                }
                __syncthreads();
                // Limit candidates in parallel, then the selection of
                // compute_limits' scan: the first push (the first candidate
                // with any, its Aitken value if it has one), the first Aitken
                // push if fewer than CMFW_MAX_LIMITS pushes precede it, and
                // the count of pushes capped at CMFW_MAX_LIMITS, as warp
                // reductions.
                const int NK = n_limit_candidates(DIM);
                int *cf = (int *)smem;  // the run products are no longer needed
                double *cla = (double *)(smem) + NK, *clr = cla + NK;
                for (int k0 = 0; k0 < NK; k0 += NT) {
                    const int k = k0 + tid;
                    int f = 0;
                    if (k < NK) {
                        double LA = 0.0, LR = 0.0;
                        f = limit_candidate(snap, snap + DD, snap + 2 * DD, DIM, k, &LA, &LR);
                        cf[k] = f;
                        cla[k] = LA;
                        clr[k] = LR;
                    }
                    const int kany = __reduce_min_sync(0xffffffffu, f ? k : 0x7fffffff);
                    const int kait = __reduce_min_sync(0xffffffffu, (f & 1) ? k : 0x7fffffff);
                    const int np = (int)__reduce_add_sync(0xffffffffu, (unsigned)__popc(f & 3));
                    if ((tid & 31) == 0) {
                        atomicMin(&s_kany, kany);
                        atomicMin(&s_kait, kait);
                        atomicAdd(&s_npush, np);
                    }
                }
                __syncthreads();
                if (s_npush > CMFW_MAX_LIMITS && s_kait != 0x7fffffff) {
                    // pushes before the first Aitken one (the cap can drop it)
                    for (int k0 = 0; k0 < NK; k0 += NT) {
                        const int k = k0 + tid;
                        const int np = (int)__reduce_add_sync(0xffffffffu, k < s_kait ? (unsigned)__popc(cf[k] & 3) : 0u);
                        if ((tid & 31) == 0) atomicAdd(&s_nbefore, np);
                    }
                    __syncthreads();
                }
                if (tid == 0) {
                    const bool have_aitken = s_kait != 0x7fffffff && s_nbefore < CMFW_MAX_LIMITS;
                    cmfw_traj_out o;
                    o.valid = 1;
                    o.n_limits = min(s_npush, CMFW_MAX_LIMITS);
                    int src = -1;
                    if (have_aitken) {
                        o.limit = cla[s_kait];
                        src = limit_source(s_kait, DIM, true);
                    } else if (s_npush > 0) {
                        const bool a1 = cf[s_kany] & 1;
                        o.limit = a1 ? cla[s_kany] : clr[s_kany];
                        src = limit_source(s_kany, DIM, a1);
                    } else {
                        o.limit = (double)NAN;
                    }
                    reduce_tail(snap, DIM, s_ls, o.limit, o);
                    W.out[t] = o;
                    if (W.status) W.status[t] = CMFW_TRAJ_OK;
                    if (W.limit_src) W.limit_src[t] = src;
                }
            }
        }
        __syncthreads();  // shared memory is reused by the next trajectory
    }
}

typedef void (*chunk_kernel_t)(ChunkArgs);

template <class A>
struct ChunkPick {
    chunk_kernel_t prefix, chunk;
    int dim;
};

template <class A>
static ChunkPick<A> pick_chunk(int p, int q, int dim) {
#define CMFW_CASE(P, Q, D)                                                                        \
    if (p == P && q == Q && dim == D)                                                             \
        return ChunkPick<A>{walk_prefix_kernel<P, Q, D>, walk_chunk_kernel<P, Q, D, A>, D};
    CMFW_FAMILY_CASES
#undef CMFW_CASE
#define CMFW_GEN(D) \
    case D: return ChunkPick<A>{walk_prefix_kernel<0, 0, D>, walk_chunk_kernel<0, 0, D, A>, D};
    switch (dim) {
        CMFW_GEN(2) CMFW_GEN(3) CMFW_GEN(4) CMFW_GEN(5) CMFW_GEN(6) CMFW_GEN(7) CMFW_GEN(8)
    }
#undef CMFW_GEN
    return ChunkPick<A>{nullptr, nullptr, 0};
}

// SMs of the current device, and per chunk kernel its dynamic shared
// memory attribute and CTAs per SM: queried once per device (a walk is
// ~0.1 ms, and each query is a runtime call on its host path).
static int device_sms() {
    static std::mutex mu;
    static int sms_of[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 148;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (sms_of[dev] == 0) {
        int sms = 148;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            sms = 148;
        }
        sms_of[dev] = sms;
    }
    return sms_of[dev];
}

struct ChunkKernelInfo {
    const void *fn;
    int dev, per_sm;
};

static cudaError_t chunk_kernel_setup(const void *fn, int threads, size_t shmem, int *per_sm) {
    static std::mutex mu;
    static std::vector<ChunkKernelInfo> known;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    for (const ChunkKernelInfo &k : known)
        if (k.fn == fn && k.dev == dev) {
            *per_sm = k.per_sm;
            return cudaSuccess;
        }
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
    if (e != cudaSuccess) return e;
    int n = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, shmem) != cudaSuccess || n < 1) {
        cudaGetLastError();
        n = 1;
    }
    known.push_back(ChunkKernelInfo{fn, dev, n});
    *per_sm = n;
    return cudaSuccess;
}

// Product slots for trajectories walked in parts: one per CTA of the
// chunk grid, which is never larger.
static int chunk_slots() { return 2 * device_sms(); }

struct ChunkLayout {
    size_t list, cost, count, parts, parts_e, parts_fail, total;
};
static ChunkLayout chunk_layout(int dim, int n, int nslots) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    ChunkLayout L;
    L.list = 0;
    L.cost = al((size_t)n * sizeof(int));
    L.count = L.cost + al((size_t)n * sizeof(int));
    L.parts = L.count + al((size_t)(1 + nslots) * sizeof(int));  // count, then arrive[nslots]
    L.parts_e = L.parts + al((size_t)nslots * 3 * dim * dim * sizeof(dd));
    L.parts_fail = L.parts_e + al((size_t)nslots * 3 * sizeof(int));
    L.total = L.parts_fail + al((size_t)nslots * sizeof(unsigned long long));
    return L;
}

// Survivor list with the survivors' costs and counter, arrival counters
// and the parts' products.
size_t chunk_scratch_bytes(int dim, int n) { return chunk_layout(dim, n, chunk_slots()).total; }

// The survivors' results of a chunked walk, gathered for the host entry
// point: index and record of each into buffers the host reads (mapped
// pinned memory), and their number.
__global__ void gather_survivors_kernel(const cmfw_traj_out *out, const int *list, const int *count,
                                        int *h_count, int *h_idx, cmfw_traj_out *h_rec) {
    const int c = *count;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *h_count = c;
    if (i < c) {
        const int t = list[i];
        h_idx[i] = t;
        h_rec[i] = out[t];
    }
}

template <class A>
static cudaError_t launch_chunk_t(const WalkArgs &W, void *scratch, int prefix_steps, cudaStream_t s,
                                  const HostGather *hg = nullptr) {
    ChunkPick<A> k = pick_chunk<A>(W.p, W.q, W.dim);
    if (!k.prefix) return cudaErrorInvalidValue;
    const int dim = W.dim, n = W.n_traj;
    const int nslots = chunk_slots();
    const ChunkLayout lay = chunk_layout(dim, n, nslots);
    char *p = (char *)scratch;
    ChunkArgs C;
    C.w = W;
    C.list = (int *)(p + lay.list);
    C.cost = (int *)(p + lay.cost);
    C.count = (int *)(p + lay.count);
    C.arrive = C.count + 1;
    C.parts = p + lay.parts;
    C.parts_e = (int *)(p + lay.parts_e);
    C.parts_fail = (unsigned long long *)(p + lay.parts_fail);
    C.nslots = nslots;
    C.part_budget = std::min(device_sms(), kMaxPartBudget);
    C.prefix_steps = prefix_steps;
    const int NT = chunk_threads(dim);
    const size_t shmem = chunk_smem_bytes<typename A::Combine::T>(dim);
    int per_sm = 1;
    cudaError_t e = chunk_kernel_setup((const void *)k.chunk, NT, shmem, &per_sm);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(C.count, 0, (size_t)(1 + nslots) * sizeof(int), s);
    if (e != cudaSuccess) return e;
    k.prefix<<<(n + kFilterThreads - 1) / kFilterThreads, kFilterThreads, 0, s>>>(C);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // persistent grid: as many CTAs as can be resident at once, at most
    // kMaxParts per trajectory and one per product slot
    long long grid = (long long)device_sms() * per_sm;
    grid = std::min<long long>(grid, (long long)std::max(n, 1) * kMaxParts);
    grid = std::min<long long>(grid, nslots);
    // launched as the filter's programmatic dependent: its CTAs may be set
    // up while the filter drains (cudaGridDependencySynchronize in the
    // kernel orders the reads)
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = shmem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (W.ev_main_start) {
        e = cudaEventRecord((cudaEvent_t)W.ev_main_start, s);
        if (e != cudaSuccess) return e;
    }
    e = cudaLaunchKernelEx(&cfg, k.chunk, C);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess && W.ev_main_stop) e = cudaEventRecord((cudaEvent_t)W.ev_main_stop, s);
    if (e != cudaSuccess || !hg) return e;
    gather_survivors_kernel<<<(n + 255) / 256, 256, 0, s>>>(W.out, C.list, C.count, hg->count, hg->idx, hg->rec);
    return cudaGetLastError();
}

// ff selects the df64 walk (float-float runs); otherwise the f64 walk with
// double-double runs, or plain FP64 runs with CMFW_F_PLAIN_RUNS.
cudaError_t launch_walk_chunked(const WalkArgs &W, bool ff, int threads, void *scratch, int prefix_steps,
                                cudaStream_t s, const HostGather *hg) {
    (void)threads;
    if (ff) return launch_chunk_t<ArithFF>(W, scratch, prefix_steps, s, hg);
    if (W.flags & CMFW_F_PLAIN_RUNS) return launch_chunk_t<ArithF64>(W, scratch, prefix_steps, s, hg);
    return launch_chunk_t<ArithDD>(W, scratch, prefix_steps, s, hg);
}

}  // namespace cmfw
