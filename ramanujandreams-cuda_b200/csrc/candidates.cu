// The delta search's candidate filter: the chunked walk's first stage (the
// singularity tests of the first lattice step, no matrix work, verdict only)
// applied to candidates of the seeded generator drawn in place, with the
// indices of the candidates that pass compacted into a list.
//
// Only the verdict is kept, so the tests run in the order that ends a
// failing candidate soonest (lattice_step_passes: inverse steps first).
// A candidate that fails here is an invalid walk whatever arithmetic walks
// it (the tests depend on the position only: cmf_pfq.cuh:164-174 lead
// coefficient, :193 denominator, :225-232 scalar solve), and it is exactly
// what the chunked walk's own filter (walk_prefix_kernel) would drop. At a
// zeta start most directions fail on their first y+ step, so the filter is
// the cheap part of a search: walking the survivors is the expensive part,
// and a proposal that ranks only the survivors competes with that.
#include <cstdio>

#include "candidates.cuh"
#include "cmfw.h"
#include "walk_arith.cuh"

namespace cmfw {
cmfw_status record_error(cmfw_status s, const char *msg);

struct FilterArgs {
    uint64_t seed;
    long long first, n;
    int lo, span;
    int p, q, dim, S;
    double z;
    double start[CMFW_MAX_AXES];
    long long *idx;
    long long cap;
    unsigned long long *count;
};

constexpr int kCandidateThreads = 128;

// The candidate's direction as the walk reads it: |d| per axis, the signs
// as a bit mask and the largest |d|; false when a component exceeds the
// walk's step cap (an invalid walk).
template <int NAX>
__device__ __forceinline__ bool candidate_axes(const FilterArgs &A, const SmallMod &mod, int naxes, long long cand,
                                               int (&absd)[NAX], uint32_t &neg, int &maxabs) {
    neg = 0;
    maxabs = 0;
    uint64_t d = 0;
#pragma unroll
    for (int a = 0; a < NAX; ++a) {
        if ((a & 3) == 0) d = candidate_draw(A.seed, cand, a >> 2);
        int v = 0;
        if (a < naxes) v = A.lo + (int)mod((uint32_t)((d >> (16 * (a & 3))) & 0xFFFFull));
        if (v < 0) neg |= 1u << a;
        absd[a] = v < 0 ? -v : v;
        maxabs = max(maxabs, absd[a]);
    }
    return maxabs <= CMFW_MAX_DIR_COMPONENT;
}

// Stages of the filter, cheapest first. Every stage only rejects
// candidates that fail one of the walk's own tests, so the survivors of
// stage 3 are exactly the candidates that pass every test:
//   1  the first test's lead coefficient (lead_verdict: rejects only when
//      the test certainly fails);
//   2  the first test in full (lead, denominator and, for an inverse step,
//      the scalar solve);
//   3  every test of the first A.S lattice steps (lattice_step_passes).
template <int STAGE, int DIM, int NAX, int PM, int QM>
__device__ __forceinline__ bool filter_stage(const FilterArgs &A, const SmallMod &mod, int naxes, const StepConst &K,
                                             long long cand) {
    int absd[NAX];
    uint32_t neg;
    int maxabs;
    if (!candidate_axes<NAX>(A, mod, naxes, cand, absd, neg, maxabs)) return false;
    double pos[NAX];
#pragma unroll
    for (int a = 0; a < NAX; ++a) pos[a] = (a < naxes) ? A.start[a] : 0.0;
    if (STAGE == 3) {
        bool ok = true;
        for (int step = 1; step <= A.S && ok; ++step)
            ok = lattice_step_passes<DIM, NAX, PM, QM>(pos, absd, neg, maxabs, K);
        return ok;
    }
    if (maxabs == 0) return true;  // no axis steps: nothing to test here
    int level, axis;
    first_tested_step<NAX>(absd, neg, K.P, level, axis);
    double at[NAX];
    position_at<NAX>(pos, absd, neg, level, axis, at);
    const bool up = !((neg >> axis) & 1u);
    if (STAGE == 1) return !step_lead_singular<DIM, NAX, PM, QM>(at, axis, up, K);
    StepMatrix<DIM> S;
    return step_matrix<false, DIM, NAX, PM, QM>(at, axis, up, K, S) == CMFW_TRAJ_OK;
}

// Almost every candidate fails its first test, and a warp runs as long as
// its longest-lived lane; so the stages run over queues in shared memory:
// stage 1 over every candidate of a block-wide slice, stage 2 over the
// stage-1 survivors and stage 3 over the stage-2 survivors, each queue
// drained a full block at a time (the rest at the end), so the lanes of a
// warp mostly do the same amount of work. Stage 1 is the hot one and its
// integer and FP64 latencies want warps in flight: five blocks per SM (96
// registers; what spills belongs to the rare stages 2 and 3) measured
// faster than four or three on an 8F7 zeta range (4.2 against 4.3 and 4.7
// ms for 10^8 candidates).
template <int P_, int Q_, int DIM>
__global__ void __launch_bounds__(kCandidateThreads, 5) filter_candidates_kernel(FilterArgs A) {
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    constexpr int T = kCandidateThreads;
    __shared__ long long q1[2 * T], q2[2 * T];
    __shared__ int n1, n2;
    const int P = (P_ > 0) ? P_ : A.p;
    const int Q = (P_ > 0) ? Q_ : A.q;
    const int naxes = P + Q;
    const StepConst K = make_step_const(P, Q, DIM, A.z);
    const SmallMod mod((uint32_t)A.span);
    if (threadIdx.x == 0) n1 = n2 = 0;
    __syncthreads();
    for (long long base = (long long)blockIdx.x * T;; base += (long long)gridDim.x * T) {
        const bool more = base < A.n;  // the same for the whole block
        if (more) {
            const long long c = base + threadIdx.x;
            if (c < A.n && filter_stage<1, DIM, NAX, PM, QM>(A, mod, naxes, K, A.first + c))
                q1[atomicAdd(&n1, 1)] = A.first + c;
        }
        __syncthreads();
        // Queue sizes stay below 2T: stage 1 adds at most T to a queue 1
        // that was drained below T, so one drain (all of it on the last
        // pass, below T then) empties it below T again; that adds at most T
        // to a queue 2 below T, which is drained until below T (empty on
        // the last pass).
        const int k1 = n1;
        if (k1 > 0 && (!more || k1 >= T)) {
            const int take = min(k1, T);
            __syncthreads();  // every thread has read n1
            if (threadIdx.x < take) {
                const long long cand = q1[k1 - take + threadIdx.x];
                if (filter_stage<2, DIM, NAX, PM, QM>(A, mod, naxes, K, cand)) q2[atomicAdd(&n2, 1)] = cand;
            }
            if (threadIdx.x == 0) n1 = k1 - take;
            __syncthreads();
        }
        for (;;) {
            const int k2 = n2;
            if (k2 == 0 || (more && k2 < T)) break;
            const int take = min(k2, T);
            __syncthreads();
            if (threadIdx.x < take) {
                const long long cand = q2[k2 - take + threadIdx.x];
                if (filter_stage<3, DIM, NAX, PM, QM>(A, mod, naxes, K, cand)) {
                    const unsigned long long at = atomicAdd(A.count, 1ull);
                    if ((long long)at < A.cap) A.idx[at] = cand;
                }
            }
            if (threadIdx.x == 0) n2 = k2 - take;
            __syncthreads();
        }
        if (!more) break;
        __syncthreads();  // every thread has read n1 before the next slice adds to it
    }
}

typedef void (*filter_kernel_t)(FilterArgs);

static filter_kernel_t pick_filter(int p, int q, int dim) {
#define CMFW_CASE(P, Q, D) \
    if (p == P && q == Q && dim == D) return filter_candidates_kernel<P, Q, D>;
    CMFW_FAMILY_CASES
#undef CMFW_CASE
    switch (dim) {
        case 2: return filter_candidates_kernel<0, 0, 2>;
        case 3: return filter_candidates_kernel<0, 0, 3>;
        case 4: return filter_candidates_kernel<0, 0, 4>;
        case 5: return filter_candidates_kernel<0, 0, 5>;
        case 6: return filter_candidates_kernel<0, 0, 6>;
        case 7: return filter_candidates_kernel<0, 0, 7>;
        case 8: return filter_candidates_kernel<0, 0, 8>;
    }
    return nullptr;
}

}  // namespace cmfw

using namespace cmfw;

extern "C" cmfw_status cmfw_filter_candidates(const cmfw_desc *desc, uint64_t seed, long long first, long long n,
                                              int lo, int hi, const double *h_start, int N, int h,
                                              int prefix_steps, long long *d_idx, long long cap,
                                              unsigned long long *d_count, void *stream) {
    cmfw_status st = cmfw_check_desc(desc);
    if (st != CMFW_OK) return st;
    if (n < 0 || first < 0 || hi < lo || !h_start || !d_count || cap < 0 || (cap > 0 && !d_idx) ||
        prefix_steps < 0)
        return record_error(CMFW_EINVAL, "bad candidate filter arguments");
    if (desc->naxes > 15) return record_error(CMFW_EINVAL, "the candidate generator draws at most 15 axes");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return record_error(CMFW_ECUDA, cudaGetErrorString(e));
    // the walk's own depth rule: with N - 2h <= 0 every walk is invalid
    if (n == 0 || N <= 0 || h <= 0 || N - 2 * h <= 0) return CMFW_OK;
    filter_kernel_t k = pick_filter(desc->p, desc->q, desc->rank);
    if (!k) return record_error(CMFW_EUNSUPPORTED, "no filter kernel for this descriptor");
    FilterArgs A;
    A.seed = seed;
    A.first = first;
    A.n = n;
    A.lo = lo;
    A.span = hi - lo + 1;
    A.p = desc->p;
    A.q = desc->q;
    A.dim = desc->rank;
    A.S = prefix_steps < N - 2 * h - 1 ? prefix_steps : N - 2 * h - 1;
    A.z = desc->z;
    for (int a = 0; a < CMFW_MAX_AXES; ++a) A.start[a] = a < desc->naxes ? h_start[a] : 0.0;
    A.idx = d_idx;
    A.cap = cap;
    A.count = d_count;
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // one resident wave: each block loops over slices of the range
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kCandidateThreads, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const long long want = (n + kCandidateThreads - 1) / kCandidateThreads;
    const long long grid = want < (long long)sms * per_sm ? want : (long long)sms * per_sm;
    k<<<(unsigned)grid, kCandidateThreads, 0, s>>>(A);
    e = cudaGetLastError();
    return e == cudaSuccess ? CMFW_OK : record_error(CMFW_ECUDA, cudaGetErrorString(e));
}
