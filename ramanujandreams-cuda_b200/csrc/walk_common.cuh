// Pieces shared by the floating-point walk kernels: the companion
// polynomial, per-row power-of-two rescaling and the matrix health test.
#pragma once

#include "cmfw_internal.cuh"

// (p, q, rank) combinations with dedicated kernels: the reference's five
// benchmark families (3F2, 4F3, 5F4, 6F5, 8F7) at the generic rank and at
// the rank reduced for z == 1 (cmf_pfq.cuh:57-59).
#define CMFW_FAMILY_CASES                                                                     \
    CMFW_CASE(3, 2, 3) CMFW_CASE(3, 2, 2) CMFW_CASE(4, 3, 4) CMFW_CASE(4, 3, 3)             \
    CMFW_CASE(5, 4, 5) CMFW_CASE(5, 4, 4) CMFW_CASE(6, 5, 6) CMFW_CASE(6, 5, 5)             \
    CMFW_CASE(8, 7, 8) CMFW_CASE(8, 7, 7)

namespace cmfw {

// Coefficients (ascending in theta) of prod_{j<n} (theta + v_j), built one
// factor at a time as in cmf_pfq.cuh:127-141; each new coefficient is
// old[k] * v + old[k-1], evaluated as one fused multiply-add.
template <int NM>
__device__ __forceinline__ void theta_product(const double (&v)[NM > 0 ? NM : 1], int n,
                                              double (&c)[NM + 1]) {
    c[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= NM; ++k) c[k] = 0.0;
#pragma unroll
    for (int j = 0; j < NM; ++j) {
        if (j < n) {
            const double x = v[j];
#pragma unroll
            for (int k = j + 1; k >= 1; --k) c[k] = __fma_rn(c[k], x, c[k - 1]);
            c[0] = c[0] * x;
        }
    }
}

// d[0..DIM] of D(theta) = theta prod(theta + y_i - 1) - z prod(theta + x_j)
// (cmf_pfq.cuh:154-162). yv already holds y_i - 1.
template <int PM, int QM, int DIM>
__device__ __forceinline__ void column_poly(const double (&xv)[PM], const double (&yv)[QM > 0 ? QM : 1],
                                            int P, int Q, double z, double (&d)[DIM + 1]) {
    double px[PM + 1], py[(QM > 0 ? QM : 0) + 1];
    theta_product<PM>(xv, P, px);
    theta_product<QM>(yv, Q, py);
#pragma unroll
    for (int k = 0; k <= DIM; ++k) {
        double a = (k <= PM && k <= P) ? -z * px[k <= PM ? k : 0] : 0.0;
        if (k >= 1 && k - 1 <= QM && k - 1 <= Q) a = a + py[(k - 1) <= QM ? (k - 1) : 0];
        d[k] = a;
    }
}

// Rescales a row by an exact power of two when its largest entry leaves
// [2^-64, 2^64); e accumulates the exponent taken out.
template <int DIM>
__device__ __forceinline__ void rescale_row(double (&row)[DIM], int &e) {
    int hm = 0;
#pragma unroll
    for (int j = 0; j < DIM; ++j) hm = max(hm, __double2hiint(row[j]) & 0x7ff00000);
    if (hm != 0 && hm < 0x7ff00000 && (hm > ((1023 + 64) << 20) || hm < ((1023 - 64) << 20))) {
        int be = min((hm >> 20) - 1023, 1022);
        const double s = __hiloint2double((1023 - be) << 20, 0);
#pragma unroll
        for (int j = 0; j < DIM; ++j) row[j] *= s;
        e += be;
    }
}

template <int DIM>
__device__ __forceinline__ bool matrix_healthy(const double (&m)[DIM][DIM]) {
    bool any_nz = false, bad = false;
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            bad |= (__double2hiint(m[r][j]) & 0x7ff00000) == 0x7ff00000;
            any_nz |= (m[r][j] != 0.0);
        }
    return any_nz && !bad;
}

}  // namespace cmfw
