// Shared device-side pieces of the CMF walk engine: parameter bundles,
// modular (Montgomery) arithmetic, float-float arithmetic, and the snapshot
// reduction that turns three walk snapshots into a result record.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cmfw.h"

#define CMFW_EPS64 2.220446049250313e-16
#define CMFW_LN2 0.69314718055994530942
#define CMFW_MAX_LIMITS 256  // cmf_walk_f64.cu:33

namespace cmfw {

// For cmfw_walk_host's chunked walks: host-readable buffers (mapped pinned
// memory, device addresses) that receive the survivors' indices, records
// and number after the walk.
struct HostGather {
    int *count, *idx;
    cmfw_traj_out *rec;
};

// Arguments common to the plain walk kernels.
struct WalkArgs {
    const cmfw_traj_in *in;
    cmfw_traj_out *out;
    uint8_t *status;   // optional
    int *limit_src;    // optional
    double *snap;      // scratch: n_traj * 3 * dim * dim doubles
    int *snap_e;       // scratch: n_traj * 3 * dim row exponents
    int n_traj, N, h;
    int p, q, dim;
    double z;
    int flags;
    void *ev_main_start, *ev_main_stop;  // optional cudaEvent_t around the main kernel (host side)
};

// ---------------------------------------------------------------------------
// Trajectory bookkeeping shared by every variant.
// ---------------------------------------------------------------------------

// Reads a trajectory's direction into |d| and sign bits and returns max|d|,
// or -1 when a component exceeds CMFW_MAX_DIR_COMPONENT.
template <int NAX>
__device__ __forceinline__ int load_direction(const cmfw_traj_in &in, int naxes, int (&absd)[NAX],
                                              uint32_t &negmask) {
    int mx = 0;
    negmask = 0;
#pragma unroll
    for (int a = 0; a < NAX; ++a) {
        int d = (a < naxes) ? in.dir[a] : 0;
        int ad = d < 0 ? -d : d;
        if (d < 0) negmask |= 1u << a;
        absd[a] = ad;
        mx = ad > mx ? ad : mx;
    }
    return mx > CMFW_MAX_DIR_COMPONENT ? -1 : mx;
}

// Axes taking a step at `level`: bit a set when |dir[a]| >= level. The walk
// visits them from the highest axis down (cmf_pfq.cuh:313-320).
template <int NAX>
__device__ __forceinline__ uint32_t level_mask(const int (&absd)[NAX], int level) {
    uint32_t m = 0;
#pragma unroll
    for (int a = 0; a < NAX; ++a) m |= (absd[a] >= level ? 1u : 0u) << a;
    return m;
}

__device__ __forceinline__ int top_axis(uint32_t mask) { return 31 - __clz(mask); }

// One direction's axis-step order in run-length form, for kernels whose
// threads all walk the same direction: the level masks change only at the
// distinct values of |dir|, so levels thr[i] .. thr[i+1]+1 all step the axes
// of mask[i] (thr[k] = 0). Held in shared memory, it keeps |dir| out of
// every thread's registers.
struct LevelPlan {
    int k;
    int thr[CMFW_MAX_AXES + 1];
    uint32_t mask[CMFW_MAX_AXES];
    uint32_t up;  // bit a set when axis a steps up (dir[a] >= 0)
    int L;        // axis steps per lattice step, sum of |dir|
};

template <int NAX>
__device__ __forceinline__ void make_level_plan(const int (&absd)[NAX], uint32_t negmask, int maxabs,
                                                LevelPlan &L) {
    int k = 0, level = maxabs;
    while (level >= 1) {
        const uint32_t m = level_mask<NAX>(absd, level);
        // the next distinct |dir| value below `level`
        int next = 0;
#pragma unroll
        for (int a = 0; a < NAX; ++a) next = (absd[a] < level && absd[a] > next) ? absd[a] : next;
        L.thr[k] = level;
        L.mask[k] = m;
        ++k;
        level = next;
    }
    L.thr[k] = 0;
    L.k = k;
    L.up = ~negmask;
    int n = 0;
    for (int i = 0; i < k; ++i) n += (L.thr[i] - L.thr[i + 1]) * __popc(L.mask[i]);
    L.L = n;
}

// ---------------------------------------------------------------------------
// Snapshot reduction (cmf_pfq.cuh:385-596 and the result selection of
// cmf_walk_f64.cu:122-153). `m` holds three dim x dim matrices (row stride
// dim) already normalised so that their largest |entry| is 1, exactly as
// the reference's snapshots are.
// ---------------------------------------------------------------------------
// Limit candidates of compute_limits (cmf_pfq.cuh:374-460), in its scan
// order: k = 0 is the primary ratio M[0][r-1] / M[1][r-1]; k >= 1 runs over
// every (column, i, j), i != j, except the primary. Each candidate pushes an
// Aitken value and/or a raw ratio, in that order.
__device__ __forceinline__ int n_limit_candidates(int dim) { return dim * dim * (dim - 1); }

__device__ __forceinline__ void candidate_index(int k, int dim, int &i, int &j, int &cc) {
    const int c = dim - 1;
    if (k == 0) {
        i = 0;
        j = 1;
        cc = c;
        return;
    }
    const int per = dim * (dim - 1);
    const int q0 = c * per;  // the primary's place in the (column, i, j) order
    const int q = (k - 1 < q0) ? k - 1 : k;
    cc = q / per;
    const int r = q % per;
    i = r / (dim - 1);
    const int jj = r % (dim - 1);
    j = jj < i ? jj : jj + 1;
}

// One candidate: flags bit 0 = Aitken pushed (value *LA), bit 1 = raw pushed (*LR).
__device__ __forceinline__ int limit_candidate(const double *m1, const double *m2, const double *m3, int dim, int k,
                                               double *LA, double *LR) {
    const double DEN_MIN = 1e-280;
    int i, j, cc;
    candidate_index(k, dim, i, j, cc);
    int flags = 0;
    const double d1 = m1[j * dim + cc], d2 = m2[j * dim + cc], d3 = m3[j * dim + cc];
    // the primary needs |q| > DEN_MIN, the others |q| >= DEN_MIN (cmf_pfq.cuh:400, 433)
    if (k == 0 ? (fabs(d1) <= DEN_MIN || fabs(d2) <= DEN_MIN || fabs(d3) <= DEN_MIN)
               : (fabs(d1) < DEN_MIN || fabs(d2) < DEN_MIN || fabs(d3) < DEN_MIN))
        return 0;
    const double r1 = m1[i * dim + cc] / d1, r2 = m2[i * dim + cc] / d2, r3 = m3[i * dim + cc] / d3;
    if (!isfinite(r1) || !isfinite(r2) || !isfinite(r3)) return 0;
    const double sc = fmax(1.0, fmax(fabs(r1), fmax(fabs(r2), fabs(r3))));
    const double den = r1 - 2.0 * r2 + r3;
    if (fabs(den) > 1e-14 * sc) {
        const double e = r2 - r3;
        const double L = r3 - e * e / den;
        // the primary's Aitken value is kept however small (cmf_pfq.cuh:410, 448)
        if (isfinite(L) && (k == 0 || fabs(L) > 1e-15)) {
            *LA = L;
            flags |= 1;
        }
    }
    if (fabs(r3) > 1e-15) {
        *LR = r3;
        flags |= 2;
    }
    return flags;
}

__device__ __forceinline__ int limit_source(int k, int dim, bool aitken) {
    int i, j, cc;
    candidate_index(k, dim, i, j, cc);
    return ((aitken ? 1 : 0) << 12) | (i << 8) | (j << 4) | cc;
}

// Folds candidate k's pushes into the running selection (first push, first
// Aitken push, count capped at CMFW_MAX_LIMITS).
struct LimitScan {
    int n = 0, src_any = -1, src_aitken = -1;
    double first_any = 0.0, first_aitken = 0.0;
    bool have_aitken = false;
    __device__ __forceinline__ void add(int flags, double LA, double LR, int k, int dim) {
        if ((flags & 1) && n < CMFW_MAX_LIMITS) {
            if (n == 0) {
                first_any = LA;
                src_any = limit_source(k, dim, true);
            }
            if (!have_aitken) {
                first_aitken = LA;
                src_aitken = limit_source(k, dim, true);
                have_aitken = true;
            }
            ++n;
        }
        if ((flags & 2) && n < CMFW_MAX_LIMITS) {
            if (n == 0) {
                first_any = LR;
                src_any = limit_source(k, dim, false);
            }
            ++n;
        }
    }
};

__device__ inline void reduce_tail(const double *m, int dim, const double *ls, double L, cmfw_traj_out &o);

__device__ inline void reduce_snapshots(const double *m, int dim, const double *ls,
                                        cmfw_traj_out &o, int *src_out) {
    const int dd = dim * dim;
    LimitScan sc;
    const int K = n_limit_candidates(dim);
    for (int k = 0; k < K; ++k) {
        double LA = 0.0, LR = 0.0;
        const int f = limit_candidate(m, m + dd, m + 2 * dd, dim, k, &LA, &LR);
        if (f) sc.add(f, LA, LR, k, dim);
    }
    o.n_limits = sc.n;
    const double L = sc.have_aitken ? sc.first_aitken : (sc.n > 0 ? sc.first_any : (double)NAN);
    o.limit = L;
    *src_out = sc.have_aitken ? sc.src_aitken : (sc.n > 0 ? sc.src_any : -1);
    reduce_tail(m, dim, ls, L, o);
}

// p, q, log_scale, precision and delta of the reduction, given the limit.
__device__ inline void reduce_tail(const double *m, int dim, const double *ls, double L, cmfw_traj_out &o) {
    const int dd = dim * dim;
    const double *m1 = m, *m2 = m + dd, *m3 = m + 2 * dd;
    const int c = dim - 1;
    double pN = m3[c], qN = m3[dim + c];
    double pNh = m2[c], qNh = m2[dim + c];
    double pN2h = m1[c], qN2h = m1[dim + c];
    o.p = pN;
    o.q = qN;
    o.log_scale = ls[2];

    // compute_precision (cmf_pfq.cuh:531-552)
    double prec = NAN;
    if (!(fabs(qN) < 1e-280 || fabs(qNh) < 1e-280)) {
        double LN = pN / qN, LNh = pNh / qNh;
        if (isfinite(LN) && isfinite(LNh)) {
            double diff = fabs(LN - LNh);
            prec = diff <= 0.0 ? (double)INFINITY : -log10(diff);
        }
    }
    o.precision = prec;

    // compute_kamidelta -> compute_delta (cmf_pfq.cuh:563-596, 476-527)
    double delta = NAN;
    if (!(fabs(qN) < 1e-280 || fabs(qNh) < 1e-280 || fabs(qN2h) < 1e-280)) {
        double LN = pN / qN, LNh = pNh / qNh, LN2h = pN2h / qN2h;
        if (isfinite(LN) && isfinite(LNh) && isfinite(LN2h)) {
            double La = NAN;
            double den = LN2h - 2.0 * LNh + LN;
            if (fabs(den) > 1e-30) {
                double e = LNh - LN;
                La = LN - e * e / den;
            }
            double Lt = isfinite(L) ? L : (isfinite(La) ? La : LN);
            // compute_delta
            double pa = pNh, qa = qNh;
            double log_q = log(fabs(qa)) + ls[1];
            if (log_q > 0.0) {
                double Lu = Lt;
                if (!isfinite(Lu)) {
                    double r1 = pN2h / qN2h, r2 = pNh / qNh, r3 = LN;
                    double dn = r1 - 2.0 * r2 + r3;
                    if (isfinite(dn) && fabs(dn) > 1e-30) {
                        double e = r2 - r3;
                        Lu = r3 - e * e / dn;
                    }
                    if (!isfinite(Lu)) Lu = LN;
                }
                if (isfinite(Lu)) {
                    double approx = pa / qa;
                    if (isfinite(approx)) {
                        double diff = fabs(Lu - approx);
                        if (diff <= 0.0) delta = INFINITY;
                        else if (isfinite(diff)) delta = -(1.0 + log(diff) / log_q);
                    }
                }
            }
        }
    }
    o.delta = delta;
}

__device__ __forceinline__ void write_invalid(const WalkArgs &W, int t, int why) {
    cmfw_traj_out o;
    o.limit = o.delta = o.p = o.q = o.precision = o.log_scale = NAN;
    o.valid = 0;
    o.n_limits = 0;
    W.out[t] = o;
    if (W.status) W.status[t] = (uint8_t)why;
    if (W.limit_src) W.limit_src[t] = -1;
}

// Reduces the three snapshots of trajectory t and writes its record.
__device__ __forceinline__ void finish_valid(const WalkArgs &W, int t, const double *snap, int dim,
                                             const double *ls) {
    cmfw_traj_out o;
    o.valid = 1;
    int src = -1;
    reduce_snapshots(snap, dim, ls, o, &src);
    W.out[t] = o;
    if (W.status) W.status[t] = CMFW_TRAJ_OK;
    if (W.limit_src) W.limit_src[t] = src;
}

// Turns rows kept with separate power-of-two exponents (value = row * 2^e)
// into the reference's snapshot form: one matrix divided by its largest
// |entry|, plus the natural log of that divisor. In place on `m`.
__device__ inline double normalise_rows(double *m, const int *e, int dim, double log_base) {
    int emax = -2147483647;
    for (int r = 0; r < dim; ++r) {
        bool nz = false;
        for (int j = 0; j < dim; ++j) nz |= (m[r * dim + j] != 0.0);
        if (nz && e[r] > emax) emax = e[r];
    }
    if (emax == -2147483647) emax = 0;
    double g = 0.0;
    for (int r = 0; r < dim; ++r) {
        int sh = e[r] - emax;
        for (int j = 0; j < dim; ++j) {
            double v = scalbn(m[r * dim + j], sh);
            m[r * dim + j] = v;
            g = fmax(g, fabs(v));
        }
    }
    if (!(g > 0.0)) return log_base + (double)emax * CMFW_LN2;
    double inv = 1.0 / g;
    for (int i = 0; i < dim * dim; ++i) m[i] *= inv;
    return log_base + (double)emax * CMFW_LN2 + log(g);
}

// ---------------------------------------------------------------------------
// Montgomery arithmetic modulo an odd m < 2^31, R = 2^32.
// x is kept as x*R mod m; sums and differences are unchanged, products go
// through REDC. Exponentiation gives the same function of the residues as
// plain (a*b) % m square-and-multiply, so Fermat-style inverses agree with
// the reference's mod_inv for every modulus, prime or not.
// ---------------------------------------------------------------------------
struct Mod {
    uint32_t m;     // modulus
    uint32_t ninv;  // -m^{-1} mod 2^32
    uint32_t r1;    // R mod m (Montgomery form of 1)
    uint32_t r2;    // R^2 mod m
};

__device__ __forceinline__ uint32_t mmul(uint32_t a, uint32_t b, const Mod &M) {
    uint64_t t = (uint64_t)a * b;
    uint32_t lo = (uint32_t)t, hi = (uint32_t)(t >> 32);
    uint32_t u = lo * M.ninv;
    uint32_t r = hi + __umulhi(u, M.m) + (lo != 0u ? 1u : 0u);
    return r >= M.m ? r - M.m : r;
}
__device__ __forceinline__ uint32_t madd(uint32_t a, uint32_t b, const Mod &M) {
    uint32_t r = a + b;
    return r >= M.m ? r - M.m : r;
}
__device__ __forceinline__ uint32_t msub(uint32_t a, uint32_t b, const Mod &M) {
    return a >= b ? a - b : a + M.m - b;
}
__device__ __forceinline__ uint32_t mto(uint32_t a, const Mod &M) { return mmul(a, M.r2, M); }
__device__ __forceinline__ uint32_t mfrom(uint32_t a, const Mod &M) { return mmul(a, 1u, M); }
// a^(m-2) in Montgomery form (left-to-right square and multiply).
__device__ __forceinline__ uint32_t minv_fermat(uint32_t a, const Mod &M) {
    uint32_t e = M.m - 2u;
    uint32_t r = M.r1;
    for (int b = 31 - __clz(e); b >= 0; --b) {
        r = mmul(r, r, M);
        if ((e >> b) & 1u) r = mmul(r, a, M);
    }
    return r;
}

// Host-side construction of a Mod record.
inline Mod make_mod_host(uint32_t m) {
    Mod M;
    M.m = m;
    uint32_t inv = 1;  // Newton iteration for m^{-1} mod 2^32
    for (int i = 0; i < 5; ++i) inv *= 2u - m * inv;
    M.ninv = (uint32_t)(0u - inv);
    M.r1 = (uint32_t)((((uint64_t)1) << 32) % m);
    M.r2 = (uint32_t)(((unsigned __int128)1 << 64) % m);
    return M;
}

// ---------------------------------------------------------------------------
// float-float arithmetic
// ---------------------------------------------------------------------------
struct ff {
    float hi, lo;
};

// double-double: hi + lo with |lo| <= ulp(hi)/2
struct dd {
    double hi, lo;
};

__device__ __forceinline__ ff ff_from(double x) {
    ff r;
    r.hi = (float)x;
    r.lo = (float)(x - (double)r.hi);
    return r;
}
__device__ __forceinline__ double ff_to(ff x) { return (double)x.hi + (double)x.lo; }

}  // namespace cmfw

namespace cmfw {
// Threads per block for a walk kernel: the caller's request (0 = 128),
// rounded down to a whole number of warps and capped by what the kernel
// was compiled for (its launch bounds), so any --block-size is accepted.
inline int clamp_block(const void *kernel, int block) {
    if (block <= 0) block = 128;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess && block > fa.maxThreadsPerBlock)
        block = fa.maxThreadsPerBlock;
    block = (block / 32) * 32;
    return block < 32 ? 32 : block;
}
}  // namespace cmfw
