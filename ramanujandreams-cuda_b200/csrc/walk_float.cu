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
#include "walk_arith.cuh"

namespace cmfw {

template <int P_, int Q_, int DIM, class A>
__global__ void __launch_bounds__(128) walk_float_kernel(WalkArgs W) {
    typedef typename A::T T;
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;  // loop bounds for the polynomials
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
    if (W.N <= 0 || W.h <= 0 || W.N - 2 * W.h <= 0) {
        write_invalid(W, t, CMFW_TRAJ_BAD_DEPTH);
        return;
    }
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
    const int cp1 = W.N - 2 * W.h, cp2 = W.N - W.h;
    double *snap = W.snap + (size_t)t * 3 * DIM * DIM;
    int *snap_e = W.snap_e + (size_t)t * 3 * DIM;
    int status = CMFW_TRAJ_OK;

    for (int step = 1; step <= W.N; ++step) {
        status = lattice_step<DIM, NAX, PM, QM, A>(m, ex, pos, absd, neg, maxabs, K);
        if (status != CMFW_TRAJ_OK) break;
        // The reference fails a step whose matrix is all zero or non-finite
        // (cmf_pfq.cuh:109); the matrix is checked once per lattice step here.
        if (!healthy<A, DIM>(m)) { status = CMFW_TRAJ_NONFINITE; break; }
        const int k = (step == cp1) ? 0 : (step == cp2) ? 1 : (step == W.N) ? 2 : -1;
        if (k >= 0) {
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
                snap_e[k * DIM + r] = ex[r];
#pragma unroll
                for (int j = 0; j < DIM; ++j) snap[(k * DIM + r) * DIM + j] = A::to(m[r][j]);
            }
        }
    }
    if (status != CMFW_TRAJ_OK) { write_invalid(W, t, status); return; }

    double ls[3];
#pragma unroll 1
    for (int k = 0; k < 3; ++k) ls[k] = normalise_rows(snap + k * DIM * DIM, snap_e + k * DIM, DIM, 0.0);
    finish_valid(W, t, snap, DIM, ls);
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
    k<<<(W.n_traj + block - 1) / block, block, 0, s>>>(W);
    return cudaGetLastError();
}

}  // namespace cmfw
