// The floating-point walk step shared by the sequential and the chunked
// kernels: arithmetic policies (FP64, float-float), one axis step
// (cmf_pfq.cuh:255-291 with the column of 146-181 and the update of
// 186-239), one lattice step (cmf_pfq.cuh:305-322), and the matrix helpers
// for products of partial walks.
//
// Representation: a walk matrix is held either with one power-of-two
// exponent per row (value = m[r][j] * 2^ex[r]; used while stepping, so a row
// is only ever rescaled by itself) or with one exponent for the whole matrix
// (used when partial walks are multiplied together).
//
// Error-free transformations (two-sum, two-product) are written with the
// explicitly rounded intrinsics (__dmul_rn, __dadd_rn, __fmul_rn, ...): the
// compiler may not contract those into fused multiply-adds, which would
// break the exactness of the error terms.
#pragma once

#include "cmfw_internal.cuh"
#include "walk_common.cuh"

namespace cmfw {

struct ArithF64;
struct ArithDD;

struct ArithF64 {
    typedef double T;
    typedef ArithF64 Combine;  // arithmetic of the products of partial walks
    static constexpr int WINDOW = 64;  // rescale outside [2^-64, 2^64)
    __device__ static __forceinline__ T from(double x) { return x; }
    __device__ static __forceinline__ double to(T x) { return x; }
    __device__ static __forceinline__ T mul(T a, T b) { return a * b; }
    __device__ static __forceinline__ T fma(T a, T b, T c) { return __fma_rn(a, b, c); }
    // products with an FP64 scalar of the step matrix (column, 1/a, ...)
    __device__ static __forceinline__ T fma_s(T a, double s, T c) { return __fma_rn(a, s, c); }
    __device__ static __forceinline__ T mul_s(T a, double s) { return a * s; }
    // a / s given inv = 1/s (rounded): the product a*inv refined by one
    // residual step, q + (a - q s) inv (Markstein), as close to the
    // correctly rounded quotient as a division
    __device__ static __forceinline__ T div_s(T a, double s, double inv) {
        const double q = __dmul_rn(a, inv);
        return __fma_rn(__fma_rn(-q, s, a), inv, q);
    }
    __device__ static __forceinline__ T neg(T a) { return -a; }
    // sum_k a[k sa] b[k sb]: the FMA chain in k order
    // sum_k a[k] s[k] for FP64 scalars s (the step matrix's column)
    template <int N>
    __device__ static __forceinline__ T dot_s(const T *a, const double *sc) {
        T x = a[0] * sc[0];
#pragma unroll
        for (int k = 1; k < N; ++k) x = __fma_rn(a[k], sc[k], x);
        return x;
    }
    template <int N>
    __device__ static __forceinline__ T dot(const T *a, int sa, const T *b, int sb) {
        T x = a[0] * b[0];
#pragma unroll
        for (int k = 1; k < N; ++k) x = __fma_rn(a[k * sa], b[k * sb], x);
        return x;
    }
    __device__ static __forceinline__ int hexp(T a) { return __double2hiint(a) & 0x7ff00000; }
    __device__ static __forceinline__ T scale(T a, int be) {
        return a * __hiloint2double((1023 - be) << 20, 0);
    }
    __device__ static __forceinline__ bool nonzero(T a) { return a != 0.0; }
    __device__ static __forceinline__ double to_combine(T a) { return a; }
};

// double-double value hi + lo (about 106 significant bits; |lo| <=
// ulp(hi)/2 after renormalisation, which fma_s and mul_s leave out) on the
// FP64 pipe. The chunked f64 walk computes its partial walks
// and their products in this arithmetic: a partial walk started from the
// identity can pass through directions that the true walk state never
// excites, and rounding those at 53 bits would be amplified when the
// partial walks are multiplied back together.
struct ArithDD {
    typedef dd T;
    typedef ArithDD Combine;
    static constexpr int WINDOW = 64;
    __device__ static __forceinline__ T from(double x) { return T{x, 0.0}; }
    __device__ static __forceinline__ double to(T x) { return __dadd_rn(x.hi, x.lo); }
    // a*b + c: FMA two-product of the high parts plus cross terms, two-sum
    // with c's high part, one fast renormalisation.
    __device__ static __forceinline__ T fma(T a, T b, T c) {
        const double p = __dmul_rn(a.hi, b.hi);
        double e = __fma_rn(a.hi, b.hi, -p);
        e = __fma_rn(a.hi, b.lo, e);
        e = __fma_rn(a.lo, b.hi, e);
        const double s = __dadd_rn(p, c.hi);
        const double bb = __dsub_rn(s, p);
        double err = __dadd_rn(__dsub_rn(p, __dsub_rn(s, bb)), __dsub_rn(c.hi, bb));
        err = __dadd_rn(err, __dadd_rn(e, c.lo));
        T r;
        r.hi = __dadd_rn(s, err);
        r.lo = __dsub_rn(err, __dsub_rn(r.hi, s));
        return r;
    }
    __device__ static __forceinline__ T mul(T a, T b) {
        const double p = __dmul_rn(a.hi, b.hi);
        double e = __fma_rn(a.hi, b.hi, -p);
        e = __fma_rn(a.hi, b.lo, e);
        e = __fma_rn(a.lo, b.hi, e);
        T r;
        r.hi = __dadd_rn(p, e);
        r.lo = __dsub_rn(e, __dsub_rn(r.hi, p));
        return r;
    }
    // a*s + c and a*s for an FP64 scalar s: one cross term fewer, and no
    // renormalisation: the pair (s, err) carries the value to double-double
    // accuracy with a low part that grows by about an ulp of the high part
    // per operation, so the runs keep their values unnormalised between
    // steps (measured: the same counts within every bar of the bench
    // batches, 4-8 % less time) and to_combine renormalises a run's product
    // for the tree
    __device__ static __forceinline__ T fma_s(T a, double sc, T c) {
        const double p = __dmul_rn(a.hi, sc);
        double e = __fma_rn(a.hi, sc, -p);
        e = __fma_rn(a.lo, sc, e);
        const double s = __dadd_rn(p, c.hi);
        const double bb = __dsub_rn(s, p);
        double err = __dadd_rn(__dsub_rn(p, __dsub_rn(s, bb)), __dsub_rn(c.hi, bb));
        err = __dadd_rn(err, __dadd_rn(e, c.lo));
        return T{s, err};
    }
    __device__ static __forceinline__ T mul_s(T a, double sc) {
        const double p = __dmul_rn(a.hi, sc);
        double e = __fma_rn(a.hi, sc, -p);
        e = __fma_rn(a.lo, sc, e);
        return T{p, e};
    }
    // a / s to double-double accuracy given inv = 1/s: the leading quotient
    // digit, the exact remainder a - q1 s, and a second digit from it
    __device__ static __forceinline__ T div_s(T a, double s, double inv) {
        const double q1 = __dmul_rn(a.hi, inv);
        const double p = __dmul_rn(q1, s);
        const double pe = __fma_rn(q1, s, -p);  // q1 s = p + pe exactly
        const double r = __dadd_rn(__dsub_rn(__dsub_rn(a.hi, p), pe), a.lo);
        const double q2 = __dmul_rn(r, inv);
        T out;
        out.hi = __dadd_rn(q1, q2);
        out.lo = __dsub_rn(q2, __dsub_rn(out.hi, q1));
        return out;
    }
    // sum_k a[k sa] b[k sb], compensated: each term's exact high product
    // and its error terms (the FMA two-product plus the cross terms) are
    // formed independently, the high parts are summed by a pairwise tree of
    // error-free two-sums whose errors join the terms' errors, and the pair
    // is renormalised once. About the work of the FMA chain, at a third of
    // its dependent depth.
    // sum_k a[k] s[k] for FP64 scalars s, compensated as dot() below
    template <int N>
    __device__ static __forceinline__ T dot_s(const T *a, const double *sc) {
        double p[N], e[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            p[k] = __dmul_rn(a[k].hi, sc[k]);
            e[k] = __fma_rn(a[k].lo, sc[k], __fma_rn(a[k].hi, sc[k], -p[k]));
        }
        return sum_pairs<N>(p, e);
    }
    // renormalised sum of N (high, error) pairs: a pairwise tree of
    // error-free two-sums over the high parts, the errors summed alongside
    template <int N>
    __device__ static __forceinline__ T sum_pairs(double (&p)[N], double (&e)[N]) {
#pragma unroll
        for (int st = 1; st < N; st <<= 1) {
#pragma unroll
            for (int k = 0; k + st < N; k += 2 * st) {
                const double s = __dadd_rn(p[k], p[k + st]);
                const double bb = __dsub_rn(s, p[k]);
                const double err = __dadd_rn(__dsub_rn(p[k], __dsub_rn(s, bb)), __dsub_rn(p[k + st], bb));
                p[k] = s;
                e[k] = __dadd_rn(__dadd_rn(e[k], e[k + st]), err);
            }
        }
        T r;
        r.hi = __dadd_rn(p[0], e[0]);
        r.lo = __dsub_rn(e[0], __dsub_rn(r.hi, p[0]));
        return r;
    }
    template <int N>
    __device__ static __forceinline__ T dot(const T *a, int sa, const T *b, int sb) {
        double p[N], e[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const T x = a[k * sa], y = b[k * sb];
            p[k] = __dmul_rn(x.hi, y.hi);
            double ek = __fma_rn(x.hi, y.hi, -p[k]);
            ek = __fma_rn(x.hi, y.lo, ek);
            e[k] = __fma_rn(x.lo, y.hi, ek);
        }
        return sum_pairs<N>(p, e);
    }
    __device__ static __forceinline__ T neg(T a) { return T{-a.hi, -a.lo}; }
    __device__ static __forceinline__ int hexp(T a) { return __double2hiint(a.hi) & 0x7ff00000; }
    __device__ static __forceinline__ T scale(T a, int be) {
        const double s = __hiloint2double((1023 - be) << 20, 0);
        return T{a.hi * s, a.lo * s};
    }
    // (an unnormalised pair can hold a non-zero value in lo alone)
    __device__ static __forceinline__ bool nonzero(T a) { return a.hi != 0.0 || a.lo != 0.0; }
    __device__ static __forceinline__ T to_combine(T a) {
        T r;
        r.hi = __dadd_rn(a.hi, a.lo);
        r.lo = __dsub_rn(a.lo, __dsub_rn(r.hi, a.hi));
        return r;
    }
};

// float-float value hi + lo, |lo| <= ulp(hi)/2.
struct ArithFF {
    typedef ff T;
    typedef ArithF64 Combine;
    static constexpr int WINDOW = 16;  // rescale outside [2^-16, 2^16): FP32 range
    __device__ static __forceinline__ T from(double x) { return ff_from(x); }
    __device__ static __forceinline__ double to(T x) { return ff_to(x); }
    // a*b + c: FMA two-product of the high parts plus cross terms, two-sum
    // with c's high part, one fast renormalisation.
    __device__ static __forceinline__ T fma(T a, T b, T c) {
        const float p = __fmul_rn(a.hi, b.hi);
        float e = __fmaf_rn(a.hi, b.hi, -p);
        e = __fmaf_rn(a.hi, b.lo, e);
        e = __fmaf_rn(a.lo, b.hi, e);
        const float s = __fadd_rn(p, c.hi);
        const float bb = __fsub_rn(s, p);
        float err = __fadd_rn(__fsub_rn(p, __fsub_rn(s, bb)), __fsub_rn(c.hi, bb));
        err = __fadd_rn(err, __fadd_rn(e, c.lo));
        T r;
        r.hi = __fadd_rn(s, err);
        r.lo = __fsub_rn(err, __fsub_rn(r.hi, s));
        return r;
    }
    __device__ static __forceinline__ T mul(T a, T b) {
        const float p = __fmul_rn(a.hi, b.hi);
        float e = __fmaf_rn(a.hi, b.hi, -p);
        e = __fmaf_rn(a.hi, b.lo, e);
        e = __fmaf_rn(a.lo, b.hi, e);
        T r;
        r.hi = __fadd_rn(p, e);
        r.lo = __fsub_rn(e, __fsub_rn(r.hi, p));
        return r;
    }
    // an FP64 scalar enters as its float-float rounding
    __device__ static __forceinline__ T fma_s(T a, double s, T c) { return fma(a, ff_from(s), c); }
    // sum_k a[k] s[k] for FP64 scalars s: the chain in k order
    template <int N>
    __device__ static __forceinline__ T dot_s(const T *a, const double *sc) {
        T x = mul_s(a[0], sc[0]);
#pragma unroll
        for (int k = 1; k < N; ++k) x = fma_s(a[k], sc[k], x);
        return x;
    }
    __device__ static __forceinline__ T mul_s(T a, double s) { return mul(a, ff_from(s)); }
    __device__ static __forceinline__ T div_s(T a, double s, double inv) {
        (void)s;
        return mul(a, ff_from(inv));
    }
    __device__ static __forceinline__ T neg(T a) { return T{-a.hi, -a.lo}; }
    // the high part's exponent field rebased to the double bias, so the
    // rescale logic is shared with ArithF64
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
    __device__ static __forceinline__ double to_combine(T a) { return ff_to(a); }
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

// healthy() over the R rows a thread holds: bit 0 = some entry non-zero,
// bit 1 = some entry non-finite (threads that share a walk combine them).
template <class A, int R, int DIM>
__device__ __forceinline__ int health_bits(const typename A::T (&m)[R][DIM]) {
    bool any_nz = false, bad = false;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            bad |= A::hexp(m[r][j]) == 0x7ff00000;
            any_nz |= A::nonzero(m[r][j]);
        }
    return (any_nz ? 1 : 0) | (bad ? 2 : 0);
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

// A trajectory position: a register array, or a thread's column of a
// shared [NAX][NT] array (SmemPos), which frees 2 * NAX registers in
// kernels whose walk state fills the register file.
template <int NT>
struct SmemPos {
    double *p;  // &array[0][thread]
    __device__ __forceinline__ double operator[](int a) const { return p[a * NT]; }
};

template <int NAX>
__device__ __forceinline__ double pos_at(const double (&pos)[NAX], int axis) {
    double v = 0.0;
#pragma unroll
    for (int a = 0; a < NAX; ++a) v = (a == axis) ? pos[a] : v;
    return v;
}
template <int NAX, int NT>
__device__ __forceinline__ double pos_at(const SmemPos<NT> &pos, int axis) {
    return pos[axis];
}
template <int NAX>
__device__ __forceinline__ void pos_move(double (&pos)[NAX], int axis, double d) {
#pragma unroll
    for (int a = 0; a < NAX; ++a) pos[a] += (a == axis) ? d : 0.0;
}
template <int NAX, int NT>
__device__ __forceinline__ void pos_move(const SmemPos<NT> &pos, int axis, double d) {
    pos.p[axis * NT] += d;
}

// Per-launch constants of the walk step.
struct StepConst {
    int P, Q;
    double z;
    bool rank_reduced_lead;    // lead coefficient is 1 - z (dim == p == q + 1)
    double lead_scale_fixed;   // max(1, |1 - z|)
};

// The position-only part of an axis step (cmf_pfq.cuh:146-181, 186-225):
// the companion column -d/lead, 1/a and, for inverse steps, the
// row-independent beta vector and scalar solve, with the reference's
// singularity tests (cmf_pfq.cuh:173, 193, 225). None of it depends on the
// walk matrix. With FULL = false only what the tests need is formed (the
// column of a forward step is skipped). Returns a cmfw_traj_status.
template <int DIM>
struct StepMatrix {
    double col[DIM];
    double inva, sd;
    bool inverse;
};

// The lead coefficient's singularity test (the one in step_matrix) without
// the rest of the column, where the lead needs only the top two
// coefficients of each theta product: dim >= p - 1 and dim >= q, which
// holds for dim = p = q + 1 and for dim = p - 1 = q. theta_product forms
// the top coefficient of prod_{j<n} (theta + v_j) as exactly 1 and the
// next as the running sum ((v_0 + v_1) + v_2) + ... (each step a fused
// multiply-add by the top coefficient 1), so both are reproduced exactly
// here; column_poly then forms -z * px[dim] + py[dim - 1], which the
// compiler may evaluate with one rounding (fused) or two. Both roundings
// are tried: returns 1 (singular) or 0 (not) when they agree, -1 when
// they disagree, the positions are not finite or the shape does not
// qualify (the caller then forms the full column).
template <int PM, int QM, int DIM>
__device__ __forceinline__ int lead_verdict(const double (&xv)[PM], const double (&yv)[QM > 0 ? QM : 1], int P,
                                            int Q, const StepConst &K) {
    if (DIM < P - 1 || DIM < Q) return -1;
    double sx = 0.0, sy = 0.0;
#pragma unroll
    for (int j = 0; j < PM; ++j)
        if (j < P) sx = (j == 0) ? xv[0] : sx + xv[j];
#pragma unroll
    for (int i = 0; i < (QM > 0 ? QM : 1); ++i)
        if (i < Q) sy = (i == 0) ? yv[0] : sy + yv[i];
    if (!isfinite(sx) || !isfinite(sy)) return -1;
    // px[dim] and py[dim - 1] (a coefficient above a product's degree is absent)
    const bool has_x = DIM <= P, has_y = DIM - 1 <= Q;
    const double X = (DIM == P) ? 1.0 : sx;
    const double Y = (DIM - 1 == Q) ? 1.0 : sy;
    double l1, l2;
    if (has_x && has_y) {
        l1 = __fma_rn(-K.z, X, Y);
        l2 = __dadd_rn(__dmul_rn(-K.z, X), Y);
    } else if (has_x) {
        l1 = l2 = __dmul_rn(-K.z, X);
    } else {
        l1 = l2 = has_y ? Y : 0.0;
    }
    double ls = K.lead_scale_fixed;
    if (!K.rank_reduced_lead) {
        ls = 1.0;
#pragma unroll
        for (int j = 0; j < PM; ++j) if (j < P) ls += fabs(xv[j]);
#pragma unroll
        for (int i = 0; i < QM; ++i) if (i < Q) ls += fabs(yv[i]);
    }
    const double t = 64.0 * CMFW_EPS64 * ls;
    const bool b1 = !isfinite(l1) || (fabs(l1) < 1.0 && fabs(l1) <= t);
    const bool b2 = !isfinite(l2) || (fabs(l2) < 1.0 && fabs(l2) <= t);
    return b1 == b2 ? (b1 ? 1 : 0) : -1;
}

template <bool FULL, int DIM, int NAX, int PM, int QM, class POS>
__device__ __forceinline__ int step_matrix(const POS &pos, int axis, bool up, const StepConst &K,
                                           StepMatrix<DIM> &S) {
    const int P = K.P, Q = K.Q;
    const bool is_x = axis < P;
    const bool inverse = is_x ? !up : up;
    S.inverse = inverse;
    // evaluation point: x- steps evaluate at x-1, y+ steps at y+1
    const double dlt = inverse ? (is_x ? -1.0 : 1.0) : 0.0;
    const double pa = pos_at<NAX>(pos, axis);
    const double denom = up ? pa : pa - 1.0;

    double xv[PM], yv[QM > 0 ? QM : 1];
#pragma unroll
    for (int j = 0; j < PM; ++j) xv[j] = (j < P) ? pos[j] + ((j == axis) ? dlt : 0.0) : 0.0;
#pragma unroll
    for (int i = 0; i < QM; ++i) yv[i] = (i < Q) ? (pos[P + i] + ((P + i == axis) ? dlt : 0.0)) - 1.0 : 0.0;
    double d[DIM + 1];
    column_poly<PM, QM, DIM>(xv, yv, P, Q, K.z, d);
    const double lead = d[DIM];
    bool lead_bad = !isfinite(lead);
    if (!lead_bad && fabs(lead) < 1.0) {
        double ls = K.lead_scale_fixed;
        if (!K.rank_reduced_lead) {
            ls = 1.0;
#pragma unroll
            for (int j = 0; j < PM; ++j) if (j < P) ls += fabs(xv[j]);
#pragma unroll
            for (int i = 0; i < QM; ++i) if (i < Q) ls += fabs(yv[i]);
        }
        lead_bad = fabs(lead) <= 64.0 * CMFW_EPS64 * ls;
    }
    if (lead_bad) return CMFW_TRAJ_SINGULAR_LEAD;
    if (!isfinite(denom) || fabs(denom) <= 64.0 * CMFW_EPS64) return CMFW_TRAJ_SINGULAR_DENOM;
    if (!FULL && !inverse) return CMFW_TRAJ_OK;
    const double il = 1.0 / lead;
    const double inva = 1.0 / denom;
    S.inva = inva;
    // col = -d / lead: the reciprocal product plus one residual correction
    // (the reference divides, cmf_pfq.cuh:177)
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
        const double c0 = __dmul_rn(-d[i], il);
        S.col[i] = __fma_rn(__fma_rn(-c0, lead, -d[i]), il, c0);
    }
    if (inverse) {
        // back-substitution in t = out[DIM-1] (cmf_pfq.cuh:207-235); beta and
        // the scalar solve do not depend on the row
        double be[DIM];
        be[DIM - 1] = 1.0;
#pragma unroll
        for (int j = DIM - 2; j >= 0; --j) be[j] = -be[j + 1] * inva;
        double db = be[0] * S.col[0];
#pragma unroll
        for (int k = 1; k < DIM; ++k) db = __fma_rn(be[k], S.col[k], db);
        const double sd = __fma_rn(db, inva, 1.0);
        const double ss = fmax(1.0, fabs(db * inva));
        if (!isfinite(sd) || fabs(sd) <= 128.0 * CMFW_EPS64 * ss) return CMFW_TRAJ_SINGULAR_SOLVE;
        S.sd = sd;
    }
    return CMFW_TRAJ_OK;
}

// True when the axis step's lead coefficient test (the first test of
// step_matrix) certainly fails, decided from lead_verdict alone; false
// when it passes or is undecided.
template <int DIM, int NAX, int PM, int QM>
__device__ __forceinline__ bool step_lead_singular(const double (&pos)[NAX], int axis, bool up, const StepConst &K) {
    const int P = K.P, Q = K.Q;
    const bool is_x = axis < P;
    const bool inverse = is_x ? !up : up;
    const double dlt = inverse ? (is_x ? -1.0 : 1.0) : 0.0;
    double xv[PM], yv[QM > 0 ? QM : 1];
#pragma unroll
    for (int j = 0; j < PM; ++j) xv[j] = (j < P) ? pos[j] + ((j == axis) ? dlt : 0.0) : 0.0;
#pragma unroll
    for (int i = 0; i < QM; ++i) yv[i] = (i < Q) ? (pos[P + i] + ((P + i == axis) ? dlt : 0.0)) - 1.0 : 0.0;
    return lead_verdict<PM, QM, DIM>(xv, yv, P, Q, K) == 1;
}

// The first test lattice_step_passes makes: the inverse steps' pass when
// there are inverse steps, else the forward steps'; within the pass, the
// highest level any of its axes reaches and the highest such axis.
template <int NAX>
__device__ __forceinline__ void first_tested_step(const int (&absd)[NAX], uint32_t neg, int P, int &level,
                                                  int &axis) {
    int li = 0, ai = -1, lf = 0, af = -1;
#pragma unroll
    for (int a = 0; a < NAX; ++a) {
        if (absd[a] == 0) continue;
        const bool up = !((neg >> a) & 1u);
        const bool inverse = (a < P) ? !up : up;
        // ascending a: ">=" keeps the highest axis at the highest level
        if (inverse) {
            if (absd[a] >= li) { li = absd[a]; ai = a; }
        } else if (absd[a] >= lf) {
            lf = absd[a];
            af = a;
        }
    }
    if (ai >= 0) {
        level = li;
        axis = ai;
    } else {
        level = lf;
        axis = af;
    }
}

// One axis step: M <- M (I + C/a) or M (I + C/a)^-1, then the position
// moves by `up ? +1 : -1` along `axis`. Returns a cmfw_traj_status.
// The rows of the walk matrix evolve independently (row r of M A is row r
// of M times A), so a thread may hold any R of them: m[R][DIM].
template <int DIM, int NAX, int PM, int QM, class A, int R, class POS>
__device__ __forceinline__ int axis_step(typename A::T (&m)[R][DIM], int (&ex)[R], POS &pos, int axis, bool up,
                                         const StepConst &K) {
    typedef typename A::T T;
    StepMatrix<DIM> S;
    const int st = step_matrix<true, DIM, NAX, PM, QM>(pos, axis, up, K, S);
    if (st != CMFW_TRAJ_OK) return st;
    const double inva = S.inva;
    if (!S.inverse) {
        // out[j] = m[j] + m[j+1]/a, last += (m . col)/a
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const T dot = A::template dot_s<DIM>(m[r], S.col);
#pragma unroll
            for (int j = 0; j < DIM - 1; ++j) m[r][j] = A::fma_s(m[r][j + 1], inva, m[r][j]);
            m[r][DIM - 1] = A::fma_s(dot, inva, m[r][DIM - 1]);
        }
    } else {
        const double isd = 1.0 / S.sd;
        const double ninva = -inva;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            T al[DIM];
            al[DIM - 1] = A::from(0.0);
            al[DIM - 2] = m[r][DIM - 2];
#pragma unroll
            for (int j = DIM - 3; j >= 0; --j) al[j] = A::fma_s(al[j + 1], ninva, m[r][j]);
            const T da = A::template dot_s<DIM - 1>(al, S.col);
            const T tt = A::div_s(A::fma_s(da, ninva, m[r][DIM - 1]), S.sd, isd);
            // beta_j = (-1/a)^(DIM-1-j), formed as in step_matrix
            double bj = 1.0;
#pragma unroll
            for (int j = DIM - 1; j >= 0; --j) {
                m[r][j] = A::fma_s(tt, bj, al[j]);
                bj = -bj * inva;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) rescale<A, DIM>(m[r], ex[r]);
    pos_move<NAX>(pos, axis, up ? 1.0 : -1.0);
    return CMFW_TRAJ_OK;
}

// One lattice displacement: levels max|dir| .. 1, axes from the highest
// down (cmf_pfq.cuh:305-322). Returns a cmfw_traj_status.
template <int DIM, int NAX, int PM, int QM, class A>
__device__ __forceinline__ int lattice_step(typename A::T (&m)[DIM][DIM], int (&ex)[DIM], double (&pos)[NAX],
                                            const int (&absd)[NAX], uint32_t neg, int maxabs,
                                            const StepConst &K) {
    for (int level = maxabs; level >= 1; --level) {
        uint32_t mask = level_mask<NAX>(absd, level);
        while (mask) {
            const int axis = top_axis(mask);
            mask &= ~(1u << axis);
            const int st = axis_step<DIM, NAX, PM, QM, A>(m, ex, pos, axis, !((neg >> axis) & 1u), K);
            if (st != CMFW_TRAJ_OK) return st;
        }
    }
    return CMFW_TRAJ_OK;
}

// The singularity tests of one lattice displacement without the matrix
// update (the steps that decide validity depend on the position only).
template <int DIM, int NAX, int PM, int QM>
__device__ __forceinline__ int lattice_step_tests(double (&pos)[NAX], const int (&absd)[NAX], uint32_t neg,
                                                  int maxabs, const StepConst &K) {
    for (int level = maxabs; level >= 1; --level) {
        uint32_t mask = level_mask<NAX>(absd, level);
        while (mask) {
            const int axis = top_axis(mask);
            mask &= ~(1u << axis);
            const bool up = !((neg >> axis) & 1u);
            StepMatrix<DIM> S;
            const int st = step_matrix<false, DIM, NAX, PM, QM>(pos, axis, up, K, S);
            if (st != CMFW_TRAJ_OK) return st;
#pragma unroll
            for (int a = 0; a < NAX; ++a) pos[a] += (a == axis) ? (up ? 1.0 : -1.0) : 0.0;
        }
    }
    return CMFW_TRAJ_OK;
}

// The position before axis step (level, axis) of a lattice step that
// starts at pos, in closed form: levels run from max|dir| down and, within
// a level, axes from the highest down (cmf_pfq.cuh:313-320), so axis a has
// moved max(0, |d_a| - level) times at earlier levels and once more at this
// level if it comes before `axis` (a > axis, |d_a| >= level). The values
// are integers, the same as stepping one axis at a time.
template <int NAX>
__device__ __forceinline__ void position_at(const double (&pos)[NAX], const int (&absd)[NAX], uint32_t neg,
                                            int level, int axis, double (&out)[NAX]) {
#pragma unroll
    for (int a = 0; a < NAX; ++a) {
        const int moved = max(0, absd[a] - level) + ((a > axis && absd[a] >= level) ? 1 : 0);
        out[a] = pos[a] + (double)(((neg >> a) & 1u) ? -moved : moved);
    }
}

// The verdict alone (pass or not, no status): every test depends on the
// position only, so the tests can run in any order. The inverse steps
// (x-, y+), which are the ones that fail at a symmetric start, are tested
// first, then the forward steps; positions in closed form. pos advances by
// the whole step when it passes.
template <int DIM, int NAX, int PM, int QM>
__device__ __forceinline__ bool lattice_step_passes(double (&pos)[NAX], const int (&absd)[NAX], uint32_t neg,
                                                    int maxabs, const StepConst &K) {
    for (int pass = 0; pass < 2; ++pass) {
        for (int level = maxabs; level >= 1; --level) {
            uint32_t mask = level_mask<NAX>(absd, level);
            while (mask) {
                const int axis = top_axis(mask);
                mask &= ~(1u << axis);
                const bool up = !((neg >> axis) & 1u);
                const bool inverse = (axis < K.P) ? !up : up;
                if (inverse != (pass == 0)) continue;
                double at[NAX];
                position_at<NAX>(pos, absd, neg, level, axis, at);
                StepMatrix<DIM> S;
                if (step_matrix<false, DIM, NAX, PM, QM>(at, axis, up, K, S) != CMFW_TRAJ_OK) return false;
            }
        }
    }
#pragma unroll
    for (int a = 0; a < NAX; ++a) pos[a] += (double)(((neg >> a) & 1u) ? -absd[a] : absd[a]);
    return true;
}

__device__ __forceinline__ StepConst make_step_const(int P, int Q, int DIM, double z) {
    StepConst K;
    K.P = P;
    K.Q = Q;
    K.z = z;
    K.rank_reduced_lead = (DIM == P && P == Q + 1);
    K.lead_scale_fixed = fmax(1.0, fabs(1.0 - z));
    return K;
}

// Rows with their own exponents -> one matrix exponent (the largest row
// exponent among non-zero rows), written in the combine arithmetic.
template <int DIM, class A>
__device__ __forceinline__ int to_matrix_exponent(const typename A::T (&m)[DIM][DIM], const int (&ex)[DIM],
                                                  typename A::Combine::T *out /* DIM*DIM */) {
    typedef typename A::Combine C;
    int emax = -0x40000000;
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        bool nz = false;
#pragma unroll
        for (int j = 0; j < DIM; ++j) nz |= A::nonzero(m[r][j]);
        if (nz) emax = max(emax, ex[r]);
    }
    if (emax == -0x40000000) emax = 0;
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        // rows more than 2^1000 below the largest flush to zero
        const int be = max(emax - ex[r], 0);
        const bool keep = be < 1000;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            typename C::T v = A::to_combine(m[r][j]);
            out[r * DIM + j] = keep ? C::scale(v, be) : C::from(0.0);
        }
    }
    return emax;
}

// C = A B for DIM x DIM row-major matrices with matrix exponents, in the
// arithmetic C_ (double or double-double). C may be A itself (each row of C
// is formed in registers from the same row of A before it is stored) but
// not B. Returns C's exponent after a power-of-two rescale that brings its
// largest entry into [1, 2).
template <int DIM, class C_>
__device__ __forceinline__ int mat_mul_exp(const typename C_::T *a, int ea, const typename C_::T *b, int eb,
                                           typename C_::T *c) {
    typedef typename C_::T T;
    int hm = 0;
#pragma unroll 1
    for (int i = 0; i < DIM; ++i) {
        T ai[DIM], acc[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) ai[k] = a[i * DIM + k];
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            T s = C_::mul(ai[0], b[j]);
#pragma unroll
            for (int k = 1; k < DIM; ++k) s = C_::fma(ai[k], b[k * DIM + j], s);
            acc[j] = s;
            hm = max(hm, C_::hexp(s));
        }
#pragma unroll
        for (int j = 0; j < DIM; ++j) c[i * DIM + j] = acc[j];
    }
    int be = 0;
    if (hm != 0 && hm < 0x7ff00000) be = (hm >> 20) - 1023;
    if (be != 0) {
#pragma unroll 1
        for (int i = 0; i < DIM * DIM; ++i) c[i] = C_::scale(c[i], be);
    }
    return ea + eb + be;
}

}  // namespace cmfw
