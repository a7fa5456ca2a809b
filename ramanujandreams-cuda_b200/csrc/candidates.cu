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

template <int P_, int Q_, int DIM>
__global__ void __launch_bounds__(kCandidateThreads) filter_candidates_kernel(FilterArgs A) {
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    const int P = (P_ > 0) ? P_ : A.p;
    const int Q = (P_ > 0) ? Q_ : A.q;
    const int naxes = P + Q;
    const StepConst K = make_step_const(P, Q, DIM, A.z);
    const SmallMod mod((uint32_t)A.span);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < A.n; c += stride) {
        const long long cand = A.first + c;
        int absd[NAX];
        uint32_t neg = 0;
        int maxabs = 0;
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
        if (maxabs > CMFW_MAX_DIR_COMPONENT) continue;  // the walk's step cap: invalid
        double pos[NAX];
#pragma unroll
        for (int a = 0; a < NAX; ++a) pos[a] = (a < naxes) ? A.start[a] : 0.0;
        bool ok = true;
        for (int step = 1; step <= A.S && ok; ++step)
            ok = lattice_step_passes<DIM, NAX, PM, QM>(pos, absd, neg, maxabs, K);
        if (!ok) continue;
        const unsigned long long at = atomicAdd(A.count, 1ull);
        if ((long long)at < A.cap) A.idx[at] = cand;
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
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (n + kCandidateThreads - 1) / kCandidateThreads;
    const long long grid = want < (long long)sms * 16 ? want : (long long)sms * 16;
    k<<<(unsigned)grid, kCandidateThreads, 0, s>>>(A);
    e = cudaGetLastError();
    return e == cudaSuccess ? CMFW_OK : record_error(CMFW_ECUDA, cudaGetErrorString(e));
}
