// df64 walk with the reference's arithmetic (cmf_walk_df64.cu), selected by
// CMFW_F_DF64_COMPAT: float-float values with single-float reciprocals of
// the denominator, of the inverse-step solve and of the normalising maximum
// (cmf_walk_df64.cu:110-113, 138-153, 184, 194, 210), a whole-matrix
// normalisation and one log() per axis step. Its results carry the
// reference's ~1e-9 relative error; the default df64 path (walk_float.cu,
// ArithFF) does not. One thread per trajectory, matrix in registers.
#include "cmfw_internal.cuh"
#include "walk_common.cuh"

namespace cmfw {
namespace compat {

// The float-float operations of cmf_walk_df64.cu:54-113, written as the same
// expressions so that the compiler treats them as it treats the reference.
__device__ __forceinline__ void two_sum(float a, float b, float &hi, float &lo) {
    hi = a + b;
    float bv = hi - a;
    lo = (a - (hi - bv)) + (b - bv);
}
__device__ __forceinline__ void two_prod(float a, float b, float &hi, float &lo) {
    hi = a * b;
    lo = __fmaf_rn(a, b, -hi);
}
__device__ __forceinline__ ff add(ff a, ff b) {
    float sh, sl;
    two_sum(a.hi, b.hi, sh, sl);
    sl += a.lo + b.lo;
    two_sum(sh, sl, sh, sl);
    return ff{sh, sl};
}
__device__ __forceinline__ ff sub(ff a, ff b) { return add(a, ff{-b.hi, -b.lo}); }
__device__ __forceinline__ ff mul(ff a, ff b) {
    float ph, pl;
    two_prod(a.hi, b.hi, ph, pl);
    pl += a.hi * b.lo + a.lo * b.hi;
    two_sum(ph, pl, ph, pl);
    return ff{ph, pl};
}
__device__ __forceinline__ ff mul_f(ff a, float b) {
    float ph, pl;
    two_prod(a.hi, b, ph, pl);
    pl += a.lo * b;
    two_sum(ph, pl, ph, pl);
    return ff{ph, pl};
}
__device__ __forceinline__ ff div_f(ff a, float b) { return mul_f(a, 1.0f / b); }
__device__ __forceinline__ bool finite(ff a) { return isfinite(a.hi) && isfinite(a.lo); }

}  // namespace compat

template <int P_, int Q_, int DIM>
__global__ void __launch_bounds__(128) walk_df64_compat_kernel(WalkArgs W) {
    using namespace compat;
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
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
    // The reference reads an unwritten snapshot when N - 2h <= 0; here that
    // case is an invalid trajectory, as in its f64 program.
    if (W.N <= 0 || W.h <= 0 || W.N - 2 * W.h <= 0) {
        write_invalid(W, t, CMFW_TRAJ_BAD_DEPTH);
        return;
    }
    double pos[NAX];
#pragma unroll
    for (int a = 0; a < NAX; ++a) pos[a] = (a < naxes) ? in.start[a] : 0.0;
    ff m[DIM][DIM];
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int j = 0; j < DIM; ++j) m[r][j] = ff_from(r == j ? 1.0 : 0.0);

    const bool rank_reduced_lead = (DIM == P && P == Q + 1);
    const double lead_scale_fixed = fmax(1.0, fabs(1.0 - z));
    const int cp1 = W.N - 2 * W.h, cp2 = W.N - W.h;
    double *snap = W.snap + (size_t)t * 3 * DIM * DIM;
    double log_scale = 0.0, ls[3] = {0.0, 0.0, 0.0};
    int status = CMFW_TRAJ_OK;
    const ff one = ff_from(1.0), zero = ff_from(0.0);

    for (int step = 1; step <= W.N && status == CMFW_TRAJ_OK; ++step) {
        for (int level = maxabs; level >= 1 && status == CMFW_TRAJ_OK; --level) {
            uint32_t mask = level_mask<NAX>(absd, level);
            while (mask) {
                const int axis = top_axis(mask);
                mask &= ~(1u << axis);
                const bool up = !((neg >> axis) & 1u);
                const bool is_x = axis < P;
                const bool inverse = is_x ? !up : up;
                const double dlt = inverse ? (is_x ? -1.0 : 1.0) : 0.0;
                double pa = 0.0;
#pragma unroll
                for (int a = 0; a < NAX; ++a) pa = (a == axis) ? pos[a] : pa;
                const double denom = up ? pa : pa - 1.0;
                // f64 column split into float-float (cmf_walk_df64.cu:163-171)
                double xv[PM], yv[QM > 0 ? QM : 1];
#pragma unroll
                for (int j = 0; j < PM; ++j) xv[j] = (j < P) ? pos[j] + ((j == axis) ? dlt : 0.0) : 0.0;
#pragma unroll
                for (int i = 0; i < QM; ++i)
                    yv[i] = (i < Q) ? (pos[P + i] + ((P + i == axis) ? dlt : 0.0)) - 1.0 : 0.0;
                double d[DIM + 1];
                column_poly<PM, QM, DIM>(xv, yv, P, Q, z, d);
                const double lead = d[DIM];
                double lsc = lead_scale_fixed;
                if (!rank_reduced_lead) {
                    lsc = 1.0;
#pragma unroll
                    for (int j = 0; j < PM; ++j) if (j < P) lsc += fabs(xv[j]);
#pragma unroll
                    for (int i = 0; i < QM; ++i) if (i < Q) lsc += fabs(yv[i]);
                }
                if (!isfinite(lead) || fabs(lead) <= 64.0 * CMFW_EPS64 * lsc) {
                    status = CMFW_TRAJ_SINGULAR_LEAD;
                    break;
                }
                ff col[DIM];
                bool colbad = false;
#pragma unroll
                for (int i = 0; i < DIM; ++i) {
                    double c = -d[i] / lead;
                    colbad |= !isfinite(c);
                    col[i] = ff_from(c);
                }
                if (colbad) { status = CMFW_TRAJ_SINGULAR_LEAD; break; }
                const ff dn = ff_from(denom);
                if (!finite(dn) || fabsf(dn.hi) <= 64.0f * 1.19e-7f) {
                    status = CMFW_TRAJ_SINGULAR_DENOM;
                    break;
                }
                const ff inva = div_f(one, dn.hi);
                ff o[DIM][DIM];
                if (!inverse) {
#pragma unroll
                    for (int r = 0; r < DIM; ++r) {
                        ff dot = zero;
#pragma unroll
                        for (int k = 0; k < DIM; ++k) dot = add(dot, mul(m[r][k], col[k]));
#pragma unroll
                        for (int j = 0; j < DIM - 1; ++j) o[r][j] = add(m[r][j], mul(m[r][j + 1], inva));
                        o[r][DIM - 1] = add(m[r][DIM - 1], mul(dot, inva));
                    }
                } else {
                    bool bad = false;
#pragma unroll
                    for (int r = 0; r < DIM; ++r) {
                        ff al[DIM], be[DIM];
                        al[DIM - 1] = zero;
                        be[DIM - 1] = one;
#pragma unroll
                        for (int j = DIM - 2; j >= 0; --j) {
                            al[j] = sub(m[r][j], mul(al[j + 1], inva));
                            be[j] = sub(zero, mul(be[j + 1], inva));
                        }
                        ff da = zero, db = zero;
#pragma unroll
                        for (int k = 0; k < DIM; ++k) {
                            da = add(da, mul(al[k], col[k]));
                            db = add(db, mul(be[k], col[k]));
                        }
                        ff sd = add(one, mul(db, inva));
                        bad |= !finite(sd) || fabsf(sd.hi) <= 1e-10f;
                        ff isd = div_f(one, sd.hi);
                        ff tt = mul(sub(m[r][DIM - 1], mul(da, inva)), isd);
#pragma unroll
                        for (int j = 0; j < DIM; ++j) o[r][j] = add(al[j], mul(be[j], tt));
                    }
                    if (bad) { status = CMFW_TRAJ_SINGULAR_SOLVE; break; }
                }
                // df64_normalize (cmf_walk_df64.cu:138-153)
                float mx = 0.0f;
#pragma unroll
                for (int r = 0; r < DIM; ++r)
#pragma unroll
                    for (int j = 0; j < DIM; ++j) mx = fmaxf(mx, fabsf(o[r][j].hi));
                if (!(mx > 0.0f) || !isfinite(mx)) { status = CMFW_TRAJ_NONFINITE; break; }
                const float inv = 1.0f / mx;
#pragma unroll
                for (int r = 0; r < DIM; ++r)
#pragma unroll
                    for (int j = 0; j < DIM; ++j) m[r][j] = mul_f(o[r][j], inv);
                log_scale += log((double)mx);
#pragma unroll
                for (int a = 0; a < NAX; ++a) pos[a] += (a == axis) ? (up ? 1.0 : -1.0) : 0.0;
            }
        }
        if (status != CMFW_TRAJ_OK) break;
        const int k = (step == cp1) ? 0 : (step == cp2) ? 1 : (step == W.N) ? 2 : -1;
        if (k >= 0) {
            ls[k] = log_scale;
#pragma unroll
            for (int r = 0; r < DIM; ++r)
#pragma unroll
                for (int j = 0; j < DIM; ++j) snap[(k * DIM + r) * DIM + j] = ff_to(m[r][j]);
        }
    }
    if (status != CMFW_TRAJ_OK) { write_invalid(W, t, status); return; }
    finish_valid(W, t, snap, DIM, ls);
}

typedef void (*walk_kernel_t)(WalkArgs);

static walk_kernel_t pick_df64_compat(int p, int q, int dim) {
#define CMFW_CASE(P, Q, D) \
    if (p == P && q == Q && dim == D) return walk_df64_compat_kernel<P, Q, D>;
    CMFW_FAMILY_CASES
#undef CMFW_CASE
    switch (dim) {
        case 2: return walk_df64_compat_kernel<0, 0, 2>;
        case 3: return walk_df64_compat_kernel<0, 0, 3>;
        case 4: return walk_df64_compat_kernel<0, 0, 4>;
        case 5: return walk_df64_compat_kernel<0, 0, 5>;
        case 6: return walk_df64_compat_kernel<0, 0, 6>;
        case 7: return walk_df64_compat_kernel<0, 0, 7>;
        case 8: return walk_df64_compat_kernel<0, 0, 8>;
    }
    return nullptr;
}

cudaError_t launch_walk_df64_compat(const WalkArgs &W, int block, cudaStream_t s) {
    walk_kernel_t k = pick_df64_compat(W.p, W.q, W.dim);
    if (!k) return cudaErrorInvalidValue;
    block = clamp_block((const void *)k, block);
    k<<<(W.n_traj + block - 1) / block, block, 0, s>>>(W);
    return cudaGetLastError();
}

}  // namespace cmfw
