// Sequential floating-point walk: one thread per trajectory, the rank x rank
// walk matrix held in registers. One kernel template serves two
// arithmetics (walk_arith.cuh):
//   ArithF64 -- native FP64 (replaces walk_kernel_f64, cmf_walk_f64.cu:94-154,
//               whose matrix lives in a 9.5 KB local-memory stack frame);
//   ArithFF  -- float-float rows on the FP32 pipe with error-free products
//               (the accurate df64 path; the reference's df64 semantics are
//               kept separately in walk_df64_compat.cu).
// The chunked walk (walk_chunked.cu) splits one trajectory over a CTA and is
// the default; this kernel is selected with CMFW_F_SEQUENTIAL.
//
// Differences of method from the reference (same mathematics; results stay
// within the tolerances the parity tests state):
//  * each row keeps its own power-of-two exponent and is rescaled only when
//    its largest entry leaves a window around 1: no per-step max/divide/log
//    over the whole matrix (cmf_pfq.cuh:100-116). At the snapshot depths the
//    rows are brought back to the reference's form (matrix / max|entry|, with
//    the natural log of the divisor accumulated), see normalise_rows().
//  * the companion column uses one reciprocal of the lead coefficient, and
//    the inverse step one reciprocal of the row-independent scalar solve.
//  * scalars shared by all rows (column, 1/a, the inverse-step beta vector
//    and solve) are formed in FP64 for both arithmetics.
// The singularity tests are the reference's (cmf_pfq.cuh:173, 193, 225).
#include "walk_seq.cuh"

namespace cmfw {

template <int P_, int Q_, int DIM, class A>
__global__ void __launch_bounds__(128) walk_float_kernel(WalkArgs W) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= W.n_traj) return;
    walk_seq_one<P_, Q_, DIM, A>(W, t, W.N, W.snap + (size_t)t * 3 * DIM * DIM, W.snap_e + (size_t)t * 3 * DIM);
}

typedef void (*walk_kernel_t)(WalkArgs);

// Kernel table: the five families the reference benchmarks, at both ranks,
// plus a generic kernel per rank for any other (p, q).
template <class A>
static walk_kernel_t pick_float(int p, int q, int dim) {
#define CMFW_CASE(P, Q, D) \
    if (p == P && q == Q && dim == D) return walk_float_kernel<P, Q, D, A>;
    CMFW_FAMILY_CASES
#undef CMFW_CASE
    switch (dim) {
        case 2: return walk_float_kernel<0, 0, 2, A>;
        case 3: return walk_float_kernel<0, 0, 3, A>;
        case 4: return walk_float_kernel<0, 0, 4, A>;
        case 5: return walk_float_kernel<0, 0, 5, A>;
        case 6: return walk_float_kernel<0, 0, 6, A>;
        case 7: return walk_float_kernel<0, 0, 7, A>;
        case 8: return walk_float_kernel<0, 0, 8, A>;
    }
    return nullptr;
}

cudaError_t launch_walk_seq(const WalkArgs &W, bool ff, int block, cudaStream_t s) {
    walk_kernel_t k = ff ? pick_float<ArithFF>(W.p, W.q, W.dim) : pick_float<ArithF64>(W.p, W.q, W.dim);
    if (!k) return cudaErrorInvalidValue;
    block = clamp_block((const void *)k, block);
    if (W.ev_main_start) cudaEventRecord((cudaEvent_t)W.ev_main_start, s);
    k<<<(W.n_traj + block - 1) / block, block, 0, s>>>(W);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && W.ev_main_stop) e = cudaEventRecord((cudaEvent_t)W.ev_main_stop, s);
    return e;
}

}  // namespace cmfw
