// Floating-point walks: one thread per trajectory, the rank x rank walk
// matrix held in registers. One kernel template serves two arithmetics:
//   ArithF64 -- native FP64 (replaces walk_kernel_f64, cmf_walk_f64.cu:94-154,
//               whose matrix lives in a 9.5 KB local-memory stack frame);
//   ArithFF  -- float-float rows on the FP32 pipe with error-free products
//               (the accurate df64 path; the reference's df64 semantics are
//               kept separately in walk_df64_compat.cu).
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
#include "cmfw_internal.cuh"
#include "walk_common.cuh"

namespace cmfw {

struct ArithF64 {
    typedef double T;
    static constexpr int WINDOW = 64;  // rescale outside [2^-64, 2^64)
    __device__ static __forceinline__ T from(double x) { return x; }
    __device__ static __forceinline__ double to(T x) { return x; }
    __device__ static __forceinline__ T mul(T a, T b) { return a * b; }
    __device__ static __forceinline__ T fma(T a, T b, T c) { return __fma_rn(a, b, c); }
    __device__ static __forceinline__ T neg(T a) { return -a; }
    __device__ static __forceinline__ int hexp(T a) { return __double2hiint(a) & 0x7ff00000; }
    __device__ static __forceinline__ T scale(T a, int be) {
        return a * __hiloint2double((1023 - be) << 20, 0);
    }
    __device__ static __forceinline__ bool nonzero(T a) { return a != 0.0; }
};

// float-float value hi + lo, |lo| <= ulp(hi)/2.
struct ArithFF {
    typedef ff T;
    static constexpr int WINDOW = 16;  // rescale outside [2^-16, 2^16): FP32 range
    __device__ static __forceinline__ T from(double x) { return ff_from(x); }
    __device__ static __forceinline__ double to(T x) { return ff_to(x); }
    // a*b + c: FMA two-product of the high parts plus cross terms, two-sum
    // with c's high part, one fast renormalisation.
    __device__ static __forceinline__ T fma(T a, T b, T c) {
        float p = a.hi * b.hi;
        float e = __fmaf_rn(a.hi, b.hi, -p);
        e = __fmaf_rn(a.hi, b.lo, e);
        e = __fmaf_rn(a.lo, b.hi, e);
        float s = p + c.hi;
        float bb = s - p;
        float err = (p - (s - bb)) + (c.hi - bb);
        err = err + (e + c.lo);
        T r;
        r.hi = s + err;
        r.lo = err - (r.hi - s);
        return r;
    }
    __device__ static __forceinline__ T mul(T a, T b) {
        float p = a.hi * b.hi;
        float e = __fmaf_rn(a.hi, b.hi, -p);
        e = __fmaf_rn(a.hi, b.lo, e);
        e = __fmaf_rn(a.lo, b.hi, e);
        T r;
        r.hi = p + e;
        r.lo = e - (r.hi - p);
        return r;
    }
    __device__ static __forceinline__ T neg(T a) { return T{-a.hi, -a.lo}; }
    // biased double-style exponent field of the high part, for the shared
    // rescale logic (float exponent rebased to the double bias).
    __device__ static __forceinline__ int hexp(T a) {
        int f = (__float_as_int(a.hi) >> 23) & 0xff;
        if (f == 0) return 0;
        if (f == 0xff) return 0x7ff00000;
        return (f - 127 + 1023) << 20;
    }
    __device__ static __forceinline__ T scale(T a, int be) {
        float s = __int_as_float((127 - be) << 23);
        return T{a.hi * s, a.lo * s};
    }
    __device__ static __forceinline__ bool nonzero(T a) { return a.hi != 0.0f; }
};

template <class A, int DIM>
__device__ __forceinline__ void rescale(typename A::T (&row)[DIM], int &e) {
    int hm = 0;
#pragma unroll
    for (int j = 0; j < DIM; ++j) hm = max(hm, A::hexp(row[j]));
    if (hm != 0 && hm < 0x7ff00000 &&
        (hm >= ((1023 + A::WINDOW) << 20) || hm < ((1023 - A::WINDOW) << 20))) {
        const int be = (hm >> 20) - 1023;
#pragma unroll
        for (int j = 0; j < DIM; ++j) row[j] = A::scale(row[j], be);
        e += be;
    }
}

template <class A, int DIM>
__device__ __forceinline__ bool healthy(const typename A::T (&m)[DIM][DIM]) {
    bool any_nz = false, bad = false;
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            bad |= A::hexp(m[r][j]) == 0x7ff00000;
            any_nz |= A::nonzero(m[r][j]);
        }
    return any_nz && !bad;
}

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
    const double z = W.z;
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

    const bool rank_reduced_lead = (DIM == P && P == Q + 1);
    const double lead_scale_fixed = fmax(1.0, fabs(1.0 - z));
    const int cp1 = W.N - 2 * W.h, cp2 = W.N - W.h;
    double *snap = W.snap + (size_t)t * 3 * DIM * DIM;
    int *snap_e = W.snap_e + (size_t)t * 3 * DIM;
    int status = CMFW_TRAJ_OK;

    for (int step = 1; step <= W.N && status == CMFW_TRAJ_OK; ++step) {
        for (int level = maxabs; level >= 1 && status == CMFW_TRAJ_OK; --level) {
            uint32_t mask = level_mask<NAX>(absd, level);
            while (mask) {
                const int axis = top_axis(mask);
                mask &= ~(1u << axis);
                const bool up = !((neg >> axis) & 1u);
                const bool is_x = axis < P;
                const bool inverse = is_x ? !up : up;
                // Evaluation point: x- steps evaluate at x-1, y+ steps at y+1
                // (cmf_pfq.cuh:264-282).
                const double dlt = inverse ? (is_x ? -1.0 : 1.0) : 0.0;
                double pa = 0.0;
#pragma unroll
                for (int a = 0; a < NAX; ++a) pa = (a == axis) ? pos[a] : pa;
                const double denom = up ? pa : pa - 1.0;

                // Companion column of D(theta) (cmf_pfq.cuh:146-181).
                double xv[PM], yv[QM > 0 ? QM : 1];
#pragma unroll
                for (int j = 0; j < PM; ++j) xv[j] = (j < P) ? pos[j] + ((j == axis) ? dlt : 0.0) : 0.0;
#pragma unroll
                for (int i = 0; i < QM; ++i)
                    yv[i] = (i < Q) ? (pos[P + i] + ((P + i == axis) ? dlt : 0.0)) - 1.0 : 0.0;
                double d[DIM + 1];
                column_poly<PM, QM, DIM>(xv, yv, P, Q, z, d);
                const double lead = d[DIM];
                bool lead_bad = !isfinite(lead);
                if (!lead_bad && fabs(lead) < 1.0) {
                    double ls = lead_scale_fixed;
                    if (!rank_reduced_lead) {
                        ls = 1.0;
#pragma unroll
                        for (int j = 0; j < PM; ++j) if (j < P) ls += fabs(xv[j]);
#pragma unroll
                        for (int i = 0; i < QM; ++i) if (i < Q) ls += fabs(yv[i]);
                    }
                    lead_bad = fabs(lead) <= 64.0 * CMFW_EPS64 * ls;
                }
                if (lead_bad) { status = CMFW_TRAJ_SINGULAR_LEAD; break; }
                if (!isfinite(denom) || fabs(denom) <= 64.0 * CMFW_EPS64) {
                    status = CMFW_TRAJ_SINGULAR_DENOM;
                    break;
                }
                const double il = 1.0 / lead;
                const double inva_d = 1.0 / denom;
                T col[DIM];
#pragma unroll
                for (int i = 0; i < DIM; ++i) col[i] = A::from(-d[i] * il);
                const T inva = A::from(inva_d);

                if (!inverse) {
                    // M <- M (I + C/a): out[j] = m[j] + m[j+1]/a, last += (m . col)/a
#pragma unroll
                    for (int r = 0; r < DIM; ++r) {
                        T dot = A::mul(m[r][0], col[0]);
#pragma unroll
                        for (int k = 1; k < DIM; ++k) dot = A::fma(m[r][k], col[k], dot);
#pragma unroll
                        for (int j = 0; j < DIM - 1; ++j) m[r][j] = A::fma(m[r][j + 1], inva, m[r][j]);
                        m[r][DIM - 1] = A::fma(dot, inva, m[r][DIM - 1]);
                    }
                } else {
                    // M <- M (I + C/a)^-1 by back-substitution in t = out[DIM-1]
                    // (cmf_pfq.cuh:207-235). beta and the scalar solve do not
                    // depend on the row and are formed once, in FP64.
                    double be_d[DIM], cold[DIM];
#pragma unroll
                    for (int i = 0; i < DIM; ++i) cold[i] = -d[i] * il;
                    be_d[DIM - 1] = 1.0;
#pragma unroll
                    for (int j = DIM - 2; j >= 0; --j) be_d[j] = -be_d[j + 1] * inva_d;
                    double db = be_d[0] * cold[0];
#pragma unroll
                    for (int k = 1; k < DIM; ++k) db = __fma_rn(be_d[k], cold[k], db);
                    const double sd = __fma_rn(db, inva_d, 1.0);
                    const double ss = fmax(1.0, fabs(db * inva_d));
                    if (!isfinite(sd) || fabs(sd) <= 128.0 * CMFW_EPS64 * ss) {
                        status = CMFW_TRAJ_SINGULAR_SOLVE;
                        break;
                    }
                    const T isd = A::from(1.0 / sd);
                    const T ninva = A::neg(inva);
                    T be[DIM];
#pragma unroll
                    for (int j = 0; j < DIM; ++j) be[j] = A::from(be_d[j]);
#pragma unroll
                    for (int r = 0; r < DIM; ++r) {
                        T al[DIM];
                        al[DIM - 1] = A::from(0.0);
                        al[DIM - 2] = m[r][DIM - 2];
#pragma unroll
                        for (int j = DIM - 3; j >= 0; --j) al[j] = A::fma(al[j + 1], ninva, m[r][j]);
                        T da = A::mul(al[0], col[0]);
#pragma unroll
                        for (int k = 1; k < DIM - 1; ++k) da = A::fma(al[k], col[k], da);
                        const T tt = A::mul(A::fma(da, ninva, m[r][DIM - 1]), isd);
#pragma unroll
                        for (int j = 0; j < DIM; ++j) m[r][j] = A::fma(be[j], tt, al[j]);
                    }
                }
#pragma unroll
                for (int r = 0; r < DIM; ++r) rescale<A, DIM>(m[r], ex[r]);
#pragma unroll
                for (int a = 0; a < NAX; ++a) pos[a] += (a == axis) ? (up ? 1.0 : -1.0) : 0.0;
            }
        }
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

cudaError_t launch_walk_f64(const WalkArgs &W, int block, cudaStream_t s) {
    walk_kernel_t k = pick_float<ArithF64>(W.p, W.q, W.dim);
    if (!k) return cudaErrorInvalidValue;
    if (block <= 0) block = 128;
    k<<<(W.n_traj + block - 1) / block, block, 0, s>>>(W);
    return cudaGetLastError();
}

cudaError_t launch_walk_ff(const WalkArgs &W, int block, cudaStream_t s) {
    walk_kernel_t k = pick_float<ArithFF>(W.p, W.q, W.dim);
    if (!k) return cudaErrorInvalidValue;
    if (block <= 0) block = 128;
    k<<<(W.n_traj + block - 1) / block, block, 0, s>>>(W);
    return cudaGetLastError();
}

}  // namespace cmfw
