// Chunked floating-point walk (default f64 / df64 path).
//
// A trajectory's walk is a product of N lattice-step matrices that depend
// only on the position, never on the accumulated product, so it can be cut
// into chunks walked independently and multiplied back together in order.
// Two kernels:
//
//  1. filter: one thread per trajectory walks the first S lattice steps in
//     plain FP64 (S = min(prefix_steps, N-2h-1)) and keeps nothing but the
//     verdict: a trajectory that fails there is written invalid with its
//     status, a survivor appends its index to a list. Most trajectories
//     that fail, fail here (zeta starts hit a singular lead coefficient on
//     their first y+ step). The step's singularity tests use the FP64
//     column, denominators and solve, which every arithmetic forms the same
//     way, so the verdict is the run arithmetic's.
//  2. chunk: clusters of 2 CTAs of NT threads (256 up to rank 6, else 128)
//     on a persistent grid that strides over the survivor list; each
//     survivor is walked by one CTA, or by both CTAs of a cluster when there
//     are fewer survivors than half the CTAs (the parts are multiplied in
//     order through distributed shared memory). Steps 1..N form three
//     segments [1, N-2h], [N-2h+1, N-h], [N-h+1, N] (the snapshot depths are
//     segment ends); each thread walks a contiguous run of lattice steps of
//     one segment with the same registers-only step as the sequential
//     kernel, the runs of a segment are multiplied in order by a
//     shared-memory tree, and the leader CTA forms the three snapshots
//     seg0, seg0 * seg1, seg0 * seg1 * seg2 and reduces them.
//
// The latency of one trajectory drops from N lattice steps to about
// N / (NP * NT) lattice steps + log2 NT matrix products; the total
// arithmetic is that of the sequential walk plus NP * NT - 1 dense rank^3
// products.
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
#include <cooperative_groups.h>

#include "walk_arith.cuh"

namespace cg = cooperative_groups;

namespace cmfw {

struct ChunkArgs {
    WalkArgs w;
    int *list;     // n_traj survivor indices
    int *count;    // survivors
    int prefix_steps;
};

template <int P_, int Q_, int DIM>
__global__ void __launch_bounds__(128) walk_prefix_kernel(ChunkArgs C) {
    typedef ArithF64 A;
    typedef typename A::T T;
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
    T m[DIM][DIM];
    int ex[DIM];
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        ex[r] = 0;
#pragma unroll
        for (int j = 0; j < DIM; ++j) m[r][j] = A::from((r == j) ? 1.0 : 0.0);
    }
    const StepConst K = make_step_const(P, Q, DIM, W.z);
    const int S = min(C.prefix_steps, W.N - 2 * W.h - 1);
    for (int step = 1; step <= S; ++step) {
        int st = lattice_step<DIM, NAX, PM, QM, A>(m, ex, pos, absd, neg, maxabs, K);
        if (st == CMFW_TRAJ_OK && !healthy<A, DIM>(m)) st = CMFW_TRAJ_NONFINITE;
        if (st != CMFW_TRAJ_OK) { write_invalid(W, t, st); return; }
    }
    C.list[atomicAdd(C.count, 1)] = t;
}

// Threads per trajectory: 256 while a thread's registers allow (ranks up to
// 6), 128 above.
__host__ __device__ constexpr int chunk_threads(int dim) { return dim <= 6 ? 256 : 128; }

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
                x[u] = CA::mul(T.a[i * DIM], T.b[j]);
#pragma unroll
                for (int k = 1; k < DIM; ++k) x[u] = CA::fma(T.a[i * DIM + k], T.b[k * DIM + j], x[u]);
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

// Dynamic shared memory of the chunk kernel: NT run products + 6 work
// matrices, their exponents, NT/2 product tasks with their maxima, and one
// region that holds the threads' positions during the runs and the
// products' staging area afterwards.
template <class CT>
__host__ __device__ constexpr size_t chunk_union_bytes(int dim, int nt) {
    return (size_t)CMFW_MAX_AXES * nt * sizeof(double) > (size_t)(nt / 2) * dim * dim * sizeof(CT)
               ? (size_t)CMFW_MAX_AXES * nt * sizeof(double)
               : (size_t)(nt / 2) * dim * dim * sizeof(CT);
}
template <class CT>
__host__ __device__ constexpr size_t chunk_union_offset(int dim, int nt) {
    return ((size_t)(nt + 6) * dim * dim * sizeof(CT) + (nt + 6) * sizeof(int) + 15) / 16 * 16 +
           (size_t)(nt / 2) * (sizeof(ProdTask<ArithF64>) + sizeof(int));
}
template <class CT>
__host__ __device__ constexpr size_t chunk_smem_bytes(int dim, int nt) {
    return (chunk_union_offset<CT>(dim, nt) + 15) / 16 * 16 + chunk_union_bytes<CT>(dim, nt);
}

// CTAs per cluster of the chunk kernel: a trajectory is walked by one CTA,
// or by both CTAs of a cluster when the survivors leave enough SMs (chosen
// on the device from the number of survivors).
constexpr int kChunkCluster = 2;

template <int P_, int Q_, int DIM, class A>
__global__ void __launch_bounds__(chunk_threads(DIM)) walk_chunk_kernel(ChunkArgs C) {
    constexpr int NT = chunk_threads(DIM);
    constexpr int CL = kChunkCluster;
    typedef typename A::T T;
    typedef typename A::Combine CA;
    typedef typename CA::T CT;
    const WalkArgs &W = C.w;
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    constexpr int DD = DIM * DIM;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CT *smem = (CT *)smem_raw;                  // NT run products + 6 work matrices
    int *sexp = (int *)(smem + (NT + 6) * DD);  // NT + 6 exponents
    ProdTask<CA> *tasks = (ProdTask<CA> *)(((uintptr_t)(sexp + NT + 6) + 15) & ~(uintptr_t)15);  // NT / 2
    int *pmax = (int *)(tasks + NT / 2);        // NT / 2
    unsigned char *ureg = smem_raw + (chunk_union_offset<CT>(DIM, NT) + 15) / 16 * 16;
    double *s_pos = (double *)ureg;             // during the runs: [NAX][NT] positions
    CT *stage = (CT *)ureg;                     // afterwards: product staging
    __shared__ int s_ntask, s_fkey, s_ok;
    __shared__ double s_ls[3];
    // earliest failing lattice step of this CTA's runs, as step * 16 + status
    __shared__ int s_fail;
    __shared__ LevelPlan s_plan;
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int tid = threadIdx.x;
    const int P = (P_ > 0) ? P_ : W.p;
    const int Q = (P_ > 0) ? Q_ : W.q;
    const int naxes = P + Q;
    const StepConst K = make_step_const(P, Q, DIM, W.z);

    // parts per trajectory: as many CTAs as the survivors leave room for
    const int count = *C.count;
    const int nclusters = gridDim.x / CL;
    const int NP = (count * CL <= (int)gridDim.x) ? CL : 1;
    const int per_cluster = CL / NP;
    const int part = crank % NP, sub = crank / NP;
    const int NTOT = NT * NP;

    // segments of lattice steps and the runs (global index g over the NP
    // CTAs) that cover them; the same for every trajectory of the launch.
    // Kept in shared memory and re-derived where needed, so that none of it
    // holds a register across the runs.
    __shared__ int s_segbase[3], s_segT[3];
    if (tid == 0) {
        const int rest = W.N;
        int T1 = (NTOT * W.h + rest / 2) / rest;
        T1 = max(1, min(T1, W.h));
        const int T2 = max(1, min(T1, W.h));
        const int T0 = NTOT - T1 - T2;
        s_segbase[0] = 0;
        s_segbase[1] = T0;
        s_segbase[2] = T0 + T1;
        s_segT[0] = T0;
        s_segT[1] = T1;
        s_segT[2] = T2;
    }
    __syncthreads();
    const int g = part * NT + tid;

    for (int round = 0;; ++round) {
        const int b0 = (round * nclusters + (int)(blockIdx.x / CL)) * per_cluster;
        if (b0 >= count) break;  // uniform over the cluster
        const int b = b0 + sub;
        const bool active = b < count;
        const int t = active ? C.list[b] : 0;
        if (tid == 0) {
            s_fail = 0x7fffffff;
            if (active) {
                int absd[NAX];
                uint32_t neg;
                const int maxabs = load_direction<NAX>(W.in[t], naxes, absd, neg);
                make_level_plan<NAX>(absd, neg, maxabs, s_plan);
            }
        }
        T m[DIM][DIM];
        int ex[DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
            ex[r] = 0;
#pragma unroll
            for (int j = 0; j < DIM; ++j) m[r][j] = A::from((r == j) ? 1.0 : 0.0);
        }
        __syncthreads();
        if (active) {
            // this thread's run [lo, hi) of lattice steps
            const int seg = g < s_segbase[1] ? 0 : (g < s_segbase[2] ? 1 : 2);
            const int Lseg = seg == 0 ? W.N - 2 * W.h : W.h;
            const int first = seg == 0 ? 1 : (seg == 1 ? W.N - 2 * W.h + 1 : W.N - W.h + 1);
            const int local = g - s_segbase[seg];
            const int lo = first + (int)(((long long)local * Lseg) / s_segT[seg]);
            const int hi = first + (int)(((long long)(local + 1) * Lseg) / s_segT[seg]);
            const cmfw_traj_in &in = W.in[t];
            const SmemPos<NT> pos{s_pos + tid};
#pragma unroll
            for (int a = 0; a < NAX; ++a) {
                const double d = (a < naxes) ? (double)in.dir[a] : 0.0;
                pos.p[a * NT] = (a < naxes) ? in.start[a] + (double)(lo - 1) * d : 0.0;
            }
            volatile int *fail = &s_fail;
            for (int step = lo; step < hi; ++step) {
                if (*fail < step * 16) break;  // an earlier step failed: this run is moot
                int st = lattice_step_plan<DIM, NAX, PM, QM, A>(m, ex, pos, s_plan, K);
                if (st == CMFW_TRAJ_OK && !healthy<A, DIM>(m)) st = CMFW_TRAJ_NONFINITE;
                if (st != CMFW_TRAJ_OK) {
                    atomicMin(&s_fail, step * 16 + st);
                    break;
                }
            }
        }
        sexp[tid] = to_matrix_exponent<DIM, A>(m, ex, smem + tid * DD);
        __syncthreads();
        // this CTA's share of its segment's runs: lrel = index among them,
        // ccnt = their number
        int lrel, ccnt;
        {
            const int seg = g < s_segbase[1] ? 0 : (g < s_segbase[2] ? 1 : 2);
            const int b0 = max(s_segbase[seg], part * NT);
            const int b1 = min(s_segbase[seg] + s_segT[seg], (part + 1) * NT);
            lrel = tid - (b0 - part * NT);
            ccnt = max(0, b1 - b0);
        }
        // in-order tree product of this CTA's runs of each segment, one
        // level at a time, every level's products spread over the CTA
        for (int stride = 1; stride < NT; stride <<= 1) {
            if (tid == 0) s_ntask = 0;
            __syncthreads();
            if (active && (lrel % (2 * stride)) == 0 && lrel + stride < ccnt) {
                const int q = atomicAdd(&s_ntask, 1);
                tasks[q] = ProdTask<CA>{smem + tid * DD, smem + (tid + stride) * DD, smem + tid * DD, sexp[tid],
                                        sexp[tid + stride], &sexp[tid]};
                pmax[q] = 0;
            }
            __syncthreads();
            const int nt = s_ntask;
            if (nt == 0) break;  // no segment has runs this far apart
            par_products<DIM, CA, NT>(tasks, nt, pmax, stage);
        }
        // every part's products and failure key are final (CTAs that walk
        // alone need no cluster barrier)
        if (NP > 1) cluster.sync();
        if (active && part == 0) {
            // the leader CTA combines the parts in order, forms the snapshots
            // and reduces them
            CT *y = smem + NT * DD, *x = y + 3 * DD;
            int *ye = sexp + NT, *xe = ye + 3;
            if (tid == 0) {
                int fkey = 0x7fffffff;
                for (int q = 0; q < NP; ++q) fkey = min(fkey, *cluster.map_shared_rank(&s_fail, crank + q));
                s_fkey = fkey;
                s_ntask = 0;
                s_ok = 1;
            }
            __syncthreads();
            if (s_fkey != 0x7fffffff) {
                if (tid == 0) write_invalid(W, t, s_fkey & 15);
            } else {
                // segment k = first part's product [* second part's product]
                if (tid < 3) {
                    const int k = tid;
                    const CT *pm[2];
                    int pe[2], np = 0;
                    for (int q = 0; q < NP; ++q) {
                        const int b0q = max(s_segbase[k], q * NT), b1q = min(s_segbase[k] + s_segT[k], (q + 1) * NT);
                        if (b1q <= b0q) continue;
                        const int slot = b0q - q * NT;
                        pm[np] = cluster.map_shared_rank(smem, crank + q) + slot * DD;
                        pe[np] = *cluster.map_shared_rank(sexp + slot, crank + q);
                        ++np;
                    }
                    if (np == 1) {
                        for (int i = 0; i < DD; ++i) y[k * DD + i] = pm[0][i];
                        ye[k] = pe[0];
                    } else {
                        const int q = atomicAdd(&s_ntask, 1);
                        tasks[q] = ProdTask<CA>{pm[0], pm[1], y + k * DD, pe[0], pe[1], &ye[k]};
                        pmax[q] = 0;
                    }
                }
                __syncthreads();
                if (s_ntask > 0) par_products<DIM, CA, NT>(tasks, s_ntask, pmax, stage);
                // snapshots: seg0, then * seg1, then * seg2
                for (int i = tid; i < DD; i += NT) x[i] = y[i];
                if (tid == 0) xe[0] = ye[0];
                __syncthreads();
                for (int k = 1; k < 3; ++k) {
                    if (tid == 0) {
                        tasks[0] = ProdTask<CA>{x + (k - 1) * DD, y + k * DD, x + k * DD, xe[k - 1], ye[k], &xe[k]};
                        pmax[0] = 0;
                    }
                    __syncthreads();
                    par_products<DIM, CA, NT>(tasks, 1, pmax, stage);
                }
                double *snap = W.snap + (size_t)t * 3 * DD;
                int *snap_e = W.snap_e + (size_t)t * 3 * DIM;
                for (int i = tid; i < 3 * DD; i += NT) {
                    const double v = CA::to(x[i]);
                    snap[i] = v;
                    if (!isfinite(v)) atomicAnd(&s_ok, 0);
                }
                if (tid < 3 * DIM) snap_e[tid] = xe[tid / DIM];
                __syncthreads();
                if (tid < 3) {
                    bool nz = false;
                    for (int i = 0; i < DD; ++i) nz |= snap[tid * DD + i] != 0.0;
                    if (!nz) atomicAnd(&s_ok, 0);
                }
                __syncthreads();
                if (!s_ok) {
                    if (tid == 0) write_invalid(W, t, CMFW_TRAJ_NONFINITE);
                } else {
                    if (tid < 3) s_ls[tid] = normalise_rows(snap + tid * DD, snap_e + tid * DIM, DIM, 0.0);
                    __syncthreads();
                    // limit candidates in parallel, then the in-order selection
                    const int K = n_limit_candidates(DIM);
                    int *cf = (int *)smem;                     // run products are no longer needed
                    double *cla = (double *)(smem) + K, *clr = cla + K;
                    for (int k = tid; k < K; k += NT) {
                        double LA = 0.0, LR = 0.0;
                        cf[k] = limit_candidate(snap, snap + DD, snap + 2 * DD, DIM, k, &LA, &LR);
                        cla[k] = LA;
                        clr[k] = LR;
                    }
                    __syncthreads();
                    if (tid == 0) {
                        LimitScan scn;
                        for (int k = 0; k < K; ++k)
                            if (cf[k]) scn.add(cf[k], cla[k], clr[k], k, DIM);
                        cmfw_traj_out o;
                        o.valid = 1;
                        o.n_limits = scn.n;
                        o.limit = scn.have_aitken ? scn.first_aitken : (scn.n > 0 ? scn.first_any : (double)NAN);
                        reduce_tail(snap, DIM, s_ls, o.limit, o);
                        W.out[t] = o;
                        if (W.status) W.status[t] = CMFW_TRAJ_OK;
                        if (W.limit_src)
                            W.limit_src[t] = scn.have_aitken ? scn.src_aitken : (scn.n > 0 ? scn.src_any : -1);
                    }
                }
            }
        }
        if (NP > 1)
            cluster.sync();  // the leader has read every part's shared memory
        else
            __syncthreads();  // shared products are reused by the next trajectory
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

// Survivor list and counter.
size_t chunk_scratch_bytes(int dim, int n) {
    (void)dim;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    return al((size_t)n * sizeof(int)) + 256;
}

template <class A>
static cudaError_t launch_chunk_t(const WalkArgs &W, void *scratch, int prefix_steps, cudaStream_t s) {
    ChunkPick<A> k = pick_chunk<A>(W.p, W.q, W.dim);
    if (!k.prefix) return cudaErrorInvalidValue;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const int dim = W.dim, n = W.n_traj;
    ChunkArgs C;
    C.w = W;
    char *p = (char *)scratch;
    C.list = (int *)p;
    p += al((size_t)n * sizeof(int));
    C.count = (int *)p;
    C.prefix_steps = prefix_steps;
    const int NT = chunk_threads(dim);
    const size_t shmem = chunk_smem_bytes<typename A::Combine::T>(dim, NT);
    cudaError_t e = cudaFuncSetAttribute((const void *)k.chunk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)shmem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(C.count, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    k.prefix<<<(n + 127) / 128, 128, 0, s>>>(C);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // persistent grid of 2-CTA clusters: as many as can be resident at once
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kChunkCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = shmem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cfg.gridDim = dim3((unsigned)(sms / kChunkCluster * kChunkCluster), 1, 1);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, (const void *)k.chunk, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        clusters = sms / kChunkCluster;
    }
    const int need = (n + kChunkCluster - 1) / kChunkCluster;  // one trajectory per CTA at most
    clusters = max(1, min(clusters, need));
    cfg.gridDim = dim3((unsigned)(clusters * kChunkCluster), 1, 1);
    e = cudaLaunchKernelEx(&cfg, k.chunk, C);
    return e != cudaSuccess ? e : cudaGetLastError();
}

// ff selects the df64 walk (float-float runs); otherwise the f64 walk with
// double-double runs, or plain FP64 runs with CMFW_F_PLAIN_RUNS.
cudaError_t launch_walk_chunked(const WalkArgs &W, bool ff, int threads, void *scratch, int prefix_steps,
                                cudaStream_t s) {
    (void)threads;
    if (ff) return launch_chunk_t<ArithFF>(W, scratch, prefix_steps, s);
    if (W.flags & CMFW_F_PLAIN_RUNS) return launch_chunk_t<ArithF64>(W, scratch, prefix_steps, s);
    return launch_chunk_t<ArithDD>(W, scratch, prefix_steps, s);
}

}  // namespace cmfw
