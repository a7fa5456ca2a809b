// The sequential walk of one trajectory by one thread (the body of the
// sequential batch kernel, walk_float.cu, and of the mixed-batch kernel,
// walk_mixed.cu).
#pragma once

#include "walk_arith.cuh"

namespace cmfw {

// One trajectory t walked from step 1 to N by the calling thread; the
// snapshot matrices and row exponents go to snap (3 * DIM * DIM) and snap_e
// (3 * DIM), then the result record is written. Shared by the batch kernel
// below and the mixed-batch kernel (walk_mixed.cu).
template <int P_, int Q_, int DIM, class A>
__device__ __forceinline__ void walk_seq_one(const WalkArgs &W, int t, int N, double *snap, int *snap_e) {
    typedef typename A::T T;
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;  // loop bounds for the polynomials
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    const int P = (P_ > 0) ? P_ : W.p;
    const int Q = (P_ > 0) ? Q_ : W.q;
    const int naxes = P + Q;
    const cmfw_traj_in &in = W.in[t];

    int absd[NAX];
    uint32_t neg;
    const int maxabs = load_direction<NAX>(in, naxes, absd, neg);
    if (maxabs < 0) { write_invalid(W, t, CMFW_TRAJ_STEP_CAP); return; }
    if (N <= 0 || W.h <= 0 || N - 2 * W.h <= 0) {
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
    const int cp1 = N - 2 * W.h, cp2 = N - W.h;
    int status = CMFW_TRAJ_OK;

    for (int step = 1; step <= N; ++step) {
        status = lattice_step<DIM, NAX, PM, QM, A>(m, ex, pos, absd, neg, maxabs, K);
        if (status != CMFW_TRAJ_OK) break;
        // The reference fails a step whose matrix is all zero or non-finite
        // (cmf_pfq.cuh:109); the matrix is checked once per lattice step here.
        if (!healthy<A, DIM>(m)) { status = CMFW_TRAJ_NONFINITE; break; }
        const int k = (step == cp1) ? 0 : (step == cp2) ? 1 : (step == N) ? 2 : -1;
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

}  // namespace cmfw

namespace cmfw {

// Whether trajectory t survives steps 1..N, decided from the singularity
// tests alone (step_matrix: lead coefficient, denominator, scalar solve --
// all functions of the position): CMFW_TRAJ_OK, or the status of the first
// failing step. A walk that passes can still fail on a non-finite or
// all-zero matrix, which the walk itself checks.
template <int P_, int Q_, int DIM>
__device__ __forceinline__ int scan_failure(const WalkArgs &W, int t, int N) {
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    const int P = (P_ > 0) ? P_ : W.p;
    const int Q = (P_ > 0) ? Q_ : W.q;
    const int naxes = P + Q;
    const cmfw_traj_in &in = W.in[t];
    int absd[NAX];
    uint32_t neg;
    const int maxabs = load_direction<NAX>(in, naxes, absd, neg);
    if (maxabs < 0) return CMFW_TRAJ_STEP_CAP;
    if (N <= 0 || W.h <= 0 || N - 2 * W.h <= 0) return CMFW_TRAJ_BAD_DEPTH;
    double pos[NAX];
#pragma unroll
    for (int a = 0; a < NAX; ++a) pos[a] = (a < naxes) ? in.start[a] : 0.0;
    const StepConst K = make_step_const(P, Q, DIM, W.z);
    for (int step = 1; step <= N; ++step) {
        const int st = lattice_step_tests<DIM, NAX, PM, QM>(pos, absd, neg, maxabs, K);
        if (st != CMFW_TRAJ_OK) return st;
    }
    return CMFW_TRAJ_OK;
}

}  // namespace cmfw
