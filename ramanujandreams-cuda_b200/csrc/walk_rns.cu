// Residue-number-system walks.
//
// 1. Compat walk (replaces walk_kernel_rns, cmf_walk_rns.cu:260-320). Bit-
//    identical residues to the reference: the same 64-entry modulus table,
//    the f64 companion column rounded to the nearest integer before
//    reduction, Fermat-exponent inverses, and every 100 steps (and at the
//    snapshot depths) a two-modulus CRT -> normalise -> re-round pass.
//    Layout: one group of L lanes per trajectory (L = next power of two of
//    the modulus count, at most 32), one or two moduli per lane, residues in
//    Montgomery form in registers. The reference keeps a 16 KB residue
//    matrix for 64 moduli per thread in local memory.
//
// 2. Exact walk (no reference counterpart). The product of the step
//    matrices is kept as rational residues modulo K true primes: every
//    division in the step (by the lead coefficient, by the axis denominator,
//    by the inverse step's scalar solve) is a modular inverse, so nothing is
//    rounded. One thread per (trajectory, prime); primes of one trajectory
//    share warps. Host code recovers p/q by CRT and rational reconstruction.
#include "cmfw_internal.cuh"
#include "walk_common.cuh"

namespace cmfw {

// Montgomery records for the compat modulus table, plus R^3 mod m for the
// 64-bit reductions; filled once per device by the host.
struct CompatTable {
    Mod mod[CMFW_MAX_COMPAT_MODULI];
    uint32_t r3[CMFW_MAX_COMPAT_MODULI];
    uint64_t inv_p0_mod_p1;  // the constant the reference recomputes per entry
};
__constant__ CompatTable c_compat;

// The reference's modulus table (cmf_walk_rns.cu:26-43), entry for entry:
// residues are compared bit for bit, so the same moduli are required. Only
// the first twelve entries are prime; the walk arithmetic is the same
// function of the residues either way.
static const uint32_t kCompatModuli[CMFW_MAX_COMPAT_MODULI] = {
    1073741789u, 1073741783u, 1073741741u, 1073741723u, 1073741717u, 1073741707u, 1073741693u,
    1073741683u, 1073741669u, 1073741657u, 1073741641u, 1073741623u, 1073741611u, 1073741597u,
    1073741587u, 1073741573u, 1073741563u, 1073741551u, 1073741537u, 1073741527u, 1073741513u,
    1073741503u, 1073741491u, 1073741477u, 1073741467u, 1073741453u, 1073741441u, 1073741427u,
    1073741413u, 1073741403u, 1073741391u, 1073741377u, 1073741363u, 1073741353u, 1073741341u,
    1073741329u, 1073741317u, 1073741307u, 1073741293u, 1073741281u, 1073741267u, 1073741257u,
    1073741243u, 1073741231u, 1073741219u, 1073741207u, 1073741193u, 1073741183u, 1073741171u,
    1073741157u, 1073741147u, 1073741137u, 1073741123u, 1073741111u, 1073741097u, 1073741087u,
    1073741077u, 1073741063u, 1073741051u, 1073741039u, 1073741027u, 1073741017u, 1073741003u,
    1073740991u};

const uint32_t *compat_moduli() { return kCompatModuli; }

cudaError_t upload_compat_table() {
    CompatTable T;
    for (int k = 0; k < CMFW_MAX_COMPAT_MODULI; ++k) {
        T.mod[k] = make_mod_host(kCompatModuli[k]);
        T.r3[k] = (uint32_t)(((unsigned __int128)T.mod[k].r2 << 32) % kCompatModuli[k]);
    }
    // Fermat inverse of p0 modulo p1 by square-and-multiply, as
    // cmf_walk_rns.cu:236-240 computes it.
    uint64_t p0 = kCompatModuli[0], p1 = kCompatModuli[1];
    uint64_t base = p0 % p1, res = 1, e = p1 - 2;
    while (e > 0) {
        if (e & 1) res = (res * base) % p1;
        base = (base * base) % p1;
        e >>= 1;
    }
    T.inv_p0_mod_p1 = res;
    return cudaMemcpyToSymbol(c_compat, &T, sizeof(T));
}

// to_mod(llround(x), m) (cmf_walk_rns.cu:62-66) in Montgomery form. Values
// outside the int64 range (undefined in the reference) take the x86-64
// conversion result, INT64_MIN, as the reference compiled for a CPU does.
__device__ __forceinline__ uint32_t mont_from_double(double x, const Mod &M, uint32_t r3) {
    long long v;
    if (fabs(x) < 9.223372036854775808e18) v = __double2ll_rz(round(x));
    else v = (long long)0x8000000000000000ULL;
    const bool negv = v < 0;
    const uint64_t mag = negv ? (uint64_t)0 - (uint64_t)v : (uint64_t)v;
    const uint32_t hi = (uint32_t)(mag >> 32), lo = (uint32_t)mag;
    // mag * R = hi * R^2 + lo * R (mod m); mmul accepts an unreduced first
    // factor below 2^32 when the second is reduced.
    uint32_t r = madd(mmul(hi, r3, M), mmul(lo, M.r2, M), M);
    return (negv && r != 0u) ? M.m - r : r;
}

// Column polynomial with selectable rounding: fused multiply-adds (nvcc's
// default contraction of the reference source) or separately rounded
// products and sums (the reference compiled for a CPU).
template <int NM>
__device__ __forceinline__ void theta_product_sel(const double (&v)[NM > 0 ? NM : 1], int n,
                                                  double (&c)[NM + 1], bool fused) {
    c[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= NM; ++k) c[k] = 0.0;
#pragma unroll
    for (int j = 0; j < NM; ++j) {
        if (j < n) {
            const double x = v[j];
#pragma unroll
            for (int k = j + 1; k >= 1; --k)
                c[k] = fused ? __fma_rn(c[k], x, c[k - 1]) : __dadd_rn(c[k - 1], __dmul_rn(c[k], x));
            c[0] = __dmul_rn(c[0], x);
        }
    }
}

// theta_companion_column (cmf_pfq.cuh:146-181) with the exact division.
template <int PM, int QM, int DIM>
__device__ __forceinline__ int compat_column(const double (&xv)[PM], const double (&yv)[QM > 0 ? QM : 1],
                                             int P, int Q, double z, bool fused, double (&col)[DIM]) {
    double px[PM + 1], py[(QM > 0 ? QM : 0) + 1];
    theta_product_sel<PM>(xv, P, px, fused);
    theta_product_sel<QM>(yv, Q, py, fused);
    double d[DIM + 1];
#pragma unroll
    for (int k = 0; k <= DIM; ++k) {
        double a = (k <= PM && k <= P) ? __dmul_rn(-z, px[k <= PM ? k : 0]) : 0.0;
        if (k >= 1 && k - 1 <= QM && k - 1 <= Q) a = __dadd_rn(a, py[(k - 1) <= QM ? (k - 1) : 0]);
        d[k] = a;
    }
    const double lead = d[DIM];
    double ls = 1.0;
    if (DIM == P && P == Q + 1) {
        ls = fmax(1.0, fabs(1.0 - z));
    } else {
#pragma unroll
        for (int j = 0; j < PM; ++j) if (j < P) ls += fabs(xv[j]);
#pragma unroll
        for (int i = 0; i < QM; ++i) if (i < Q) ls += fabs(yv[i]);
    }
    if (!isfinite(lead) || fabs(lead) <= 64.0 * CMFW_EPS64 * ls) return 0;
    bool ok = true;
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
        col[i] = -d[i] / lead;
        ok &= isfinite(col[i]);
    }
    return ok ? 1 : 0;
}

struct RnsArgs {
    WalkArgs w;
    int n_primes;
    int lanes;       // lanes per trajectory (power of two, <= 32)
    int trace_steps; // > 0: stop after this many steps and dump residues
    uint32_t *trace_res;
    int *trace_ok;
};

// Signed two-modulus CRT of cmf_walk_rns.cu:232-244, with the reference's
// unsigned 64-bit wrap-around kept.
__device__ __forceinline__ double crt2(uint32_t r0, uint32_t r1) {
    const uint64_t p0 = c_compat.mod[0].m, p1 = c_compat.mod[1].m;
    uint64_t diff = (r1 >= r0) ? (uint64_t)(r1 - r0) : ((uint64_t)r1 + p1 - r0);
    uint64_t t = (diff * c_compat.inv_p0_mod_p1) % p1;
    uint64_t val = r0 + p0 * t;
    uint64_t half = (p0 * p1) / 2;
    return (val > half) ? -(double)(p0 * p1 - val) : (double)val;
}

template <int P_, int Q_, int DIM, int KPL>
__global__ void __launch_bounds__(128) walk_rns_compat_kernel(RnsArgs R) {
    const WalkArgs &W = R.w;
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    const int L = R.lanes;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = gtid / L;
    const int lane = gtid % L;  // lane within the trajectory's group
    if (t >= W.n_traj) return;  // whole groups leave together (L divides 32)
    const int wl = threadIdx.x & 31;
    const unsigned gmask = (L == 32) ? 0xffffffffu : (((1u << L) - 1u) << (wl - lane));
    const int P = (P_ > 0) ? P_ : W.p;
    const int Q = (P_ > 0) ? Q_ : W.q;
    const int naxes = P + Q;
    const double z = W.z;
    const bool fused = !(W.flags & CMFW_F_UNFUSED_COLUMN);
    const cmfw_traj_in &in = W.in[t];
    const int K = R.n_primes;

    int absd[NAX];
    uint32_t neg;
    const int maxabs = load_direction<NAX>(in, naxes, absd, neg);
    const bool tracing = R.trace_steps > 0;
    const int last_step = tracing ? R.trace_steps : W.N;
    int status = CMFW_TRAJ_OK;
    if (maxabs < 0) status = CMFW_TRAJ_STEP_CAP;
    else if (!tracing && (W.N <= 0 || W.h <= 0 || W.N - 2 * W.h <= 0)) status = CMFW_TRAJ_BAD_DEPTH;

    // This lane's moduli: k = lane + 32 * s.
    Mod md[KPL];
    uint32_t r3[KPL];
    bool act[KPL];
#pragma unroll
    for (int s = 0; s < KPL; ++s) {
        const int k = lane + 32 * s;
        act[s] = k < K;
        md[s] = c_compat.mod[act[s] ? k : 0];
        r3[s] = c_compat.r3[act[s] ? k : 0];
    }
    uint32_t m[KPL][DIM][DIM];
#pragma unroll
    for (int s = 0; s < KPL; ++s)
#pragma unroll
        for (int i = 0; i < DIM; ++i)
#pragma unroll
            for (int j = 0; j < DIM; ++j) m[s][i][j] = (i == j) ? md[s].r1 : 0u;

    double pos[NAX];
#pragma unroll
    for (int a = 0; a < NAX; ++a) pos[a] = (a < naxes) ? in.start[a] : 0.0;
    const int cp1 = W.N - 2 * W.h, cp2 = W.N - W.h;
    double *snap = W.snap + (size_t)t * 3 * DIM * DIM;
    double log_scale = 0.0, ls[3] = {0.0, 0.0, 0.0};

    for (int step = 1; step <= last_step && status == CMFW_TRAJ_OK; ++step) {
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
                double xv[PM], yv[QM > 0 ? QM : 1];
#pragma unroll
                for (int j = 0; j < PM; ++j) xv[j] = (j < P) ? pos[j] + ((j == axis) ? dlt : 0.0) : 0.0;
#pragma unroll
                for (int i = 0; i < QM; ++i)
                    yv[i] = (i < Q) ? (pos[P + i] + ((P + i == axis) ? dlt : 0.0)) - 1.0 : 0.0;
                double col[DIM];
                if (!compat_column<PM, QM, DIM>(xv, yv, P, Q, z, fused, col)) {
                    status = CMFW_TRAJ_SINGULAR_LEAD;
                    break;
                }
                if (!isfinite(denom) || fabs(denom) <= 64.0 * CMFW_EPS64) {
                    status = CMFW_TRAJ_SINGULAR_DENOM;
                    break;
                }
                bool fail = false;
#pragma unroll
                for (int s = 0; s < KPL; ++s) {
                    const Mod &M = md[s];
                    uint32_t cr[DIM];
#pragma unroll
                    for (int i = 0; i < DIM; ++i) cr[i] = mont_from_double(col[i], M, r3[s]);
                    const uint32_t inva = minv_fermat(mont_from_double(denom, M, r3[s]), M);
                    if (!inverse) {
                        // cmf_walk_rns.cu:143-153
#pragma unroll
                        for (int r = 0; r < DIM; ++r) {
                            uint32_t dot = 0;
#pragma unroll
                            for (int i = 0; i < DIM; ++i) dot = madd(dot, mmul(m[s][r][i], cr[i], M), M);
#pragma unroll
                            for (int j = 0; j < DIM - 1; ++j)
                                m[s][r][j] = madd(m[s][r][j], mmul(m[s][r][j + 1], inva, M), M);
                            m[s][r][DIM - 1] = madd(m[s][r][DIM - 1], mmul(dot, inva, M), M);
                        }
                    } else {
                        // cmf_walk_rns.cu:155-178; beta, its dot product and
                        // the solve are the same for every row.
                        uint32_t be[DIM];
                        be[DIM - 1] = M.r1;
#pragma unroll
                        for (int j = DIM - 2; j >= 0; --j) be[j] = msub(0u, mmul(be[j + 1], inva, M), M);
                        uint32_t db = 0;
#pragma unroll
                        for (int i = 0; i < DIM; ++i) db = madd(db, mmul(be[i], cr[i], M), M);
                        const uint32_t sd = madd(M.r1, mmul(db, inva, M), M);
                        if (sd == 0u) fail |= act[s];
                        const uint32_t isd = minv_fermat(sd, M);
#pragma unroll
                        for (int r = 0; r < DIM; ++r) {
                            uint32_t al[DIM];
                            al[DIM - 1] = 0u;
#pragma unroll
                            for (int j = DIM - 2; j >= 0; --j) al[j] = msub(m[s][r][j], mmul(al[j + 1], inva, M), M);
                            uint32_t da = 0;
#pragma unroll
                            for (int i = 0; i < DIM; ++i) da = madd(da, mmul(al[i], cr[i], M), M);
                            const uint32_t tt = mmul(msub(m[s][r][DIM - 1], mmul(da, inva, M), M), isd, M);
#pragma unroll
                            for (int j = 0; j < DIM; ++j) m[s][r][j] = madd(al[j], mmul(be[j], tt, M), M);
                        }
                    }
                }
                if (__any_sync(gmask, fail)) { status = CMFW_TRAJ_SINGULAR_SOLVE; break; }
#pragma unroll
                for (int a = 0; a < NAX; ++a) pos[a] += (a == axis) ? (up ? 1.0 : -1.0) : 0.0;
            }
        }
        if (status != CMFW_TRAJ_OK) break;
        if (step % 100 == 0 || step == cp1 || step == cp2 || step == W.N) {
            // rns_to_double (cmf_walk_rns.cu:225-251) on the first two
            // moduli, held by lanes 0 and 1, then normalise and re-reduce.
            double mx = 0.0;
            for (int pass = 0; pass < 2; ++pass) {
                const double inv = (pass == 1 && mx > 0.0 && isfinite(mx)) ? 1.0 / mx : 1.0;
                const bool scale = pass == 1 && mx > 0.0 && isfinite(mx);
                const int k = (step == cp1) ? 0 : (step == cp2) ? 1 : (step == W.N) ? 2 : -1;
#pragma unroll
                for (int i = 0; i < DIM; ++i)
#pragma unroll
                    for (int j = 0; j < DIM; ++j) {
                        const uint32_t own = mfrom(m[0][i][j], md[0]);
                        const uint32_t r0 = __shfl_sync(gmask, own, 0, L);
                        const uint32_t r1 = __shfl_sync(gmask, own, 1, L);
                        double v = (K >= 2) ? crt2(r0, r1) : (double)r0;
                        if (pass == 0) {
                            const double x = fabs(v);
                            if (x > mx) mx = x;
                        } else {
                            if (scale) v *= inv;
                            if (k >= 0 && lane == 0 && !tracing) snap[(k * DIM + i) * DIM + j] = v;
#pragma unroll
                            for (int s = 0; s < KPL; ++s) m[s][i][j] = mont_from_double(v, md[s], r3[s]);
                        }
                    }
                if (pass == 1) {
                    if (scale) log_scale += log(mx);
                    if (k >= 0) ls[k] = log_scale;
                }
            }
        }
    }
    if (tracing) {
#pragma unroll
        for (int s = 0; s < KPL; ++s) {
            const int k = lane + 32 * s;
            if (k < K)
#pragma unroll
                for (int i = 0; i < DIM; ++i)
#pragma unroll
                    for (int j = 0; j < DIM; ++j)
                        R.trace_res[(((size_t)t * K + k) * DIM + i) * DIM + j] = mfrom(m[s][i][j], md[s]);
        }
        if (lane == 0) R.trace_ok[t] = (status == CMFW_TRAJ_OK) ? 1 : 0;
        return;
    }
    if (lane != 0) return;
    if (status != CMFW_TRAJ_OK) { write_invalid(W, t, status); return; }
    finish_valid(W, t, snap, DIM, ls);
}

typedef void (*rns_kernel_t)(RnsArgs);

template <int KPL>
static rns_kernel_t pick_rns(int p, int q, int dim) {
#define CMFW_CASE(P, Q, D) \
    if (p == P && q == Q && dim == D) return walk_rns_compat_kernel<P, Q, D, KPL>;
    CMFW_FAMILY_CASES
#undef CMFW_CASE
    switch (dim) {
        case 2: return walk_rns_compat_kernel<0, 0, 2, KPL>;
        case 3: return walk_rns_compat_kernel<0, 0, 3, KPL>;
        case 4: return walk_rns_compat_kernel<0, 0, 4, KPL>;
        case 5: return walk_rns_compat_kernel<0, 0, 5, KPL>;
        case 6: return walk_rns_compat_kernel<0, 0, 6, KPL>;
        case 7: return walk_rns_compat_kernel<0, 0, 7, KPL>;
        case 8: return walk_rns_compat_kernel<0, 0, 8, KPL>;
    }
    return nullptr;
}

cudaError_t launch_walk_rns(const WalkArgs &W, int n_primes, int trace_steps, uint32_t *trace_res,
                            int *trace_ok, int block, cudaStream_t s) {
    RnsArgs R;
    R.w = W;
    R.n_primes = n_primes;
    int L = 1;
    while (L < n_primes && L < 32) L <<= 1;
    R.lanes = L;
    R.trace_steps = trace_steps;
    R.trace_res = trace_res;
    R.trace_ok = trace_ok;
    rns_kernel_t k = (n_primes > 32) ? pick_rns<2>(W.p, W.q, W.dim) : pick_rns<1>(W.p, W.q, W.dim);
    if (!k) return cudaErrorInvalidValue;
    block = clamp_block((const void *)k, block);
    const long long threads = (long long)W.n_traj * L;
    k<<<(unsigned)((threads + block - 1) / block), block, 0, s>>>(R);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Exact walk
// ---------------------------------------------------------------------------

struct ExactArgs {
    const cmfw_traj_in *in;
    const uint32_t *primes;
    uint32_t *res;       // n_traj * 3 * 2 * K
    uint8_t *prime_ok;   // n_traj * K
    const int *pairs;    // optional (i << 8) | (j << 4) | c per trajectory
    int n_traj, N, h, K;
    int p, q, dim;
    long long zn, zd;    // z = zn / zd exactly
};

__device__ __forceinline__ uint32_t mont_from_i64(long long v, const Mod &M) {
    const bool negv = v < 0;
    const uint64_t mag = negv ? (uint64_t)0 - (uint64_t)v : (uint64_t)v;
    const uint32_t r3 = mmul(M.r2, M.r2, M);  // R^3 mod m in Montgomery form = R^2 * R^2 / R
    uint32_t r = madd(mmul((uint32_t)(mag >> 32), r3, M), mmul((uint32_t)mag, M.r2, M), M);
    return (negv && r != 0u) ? M.m - r : r;
}

template <int P_, int Q_, int DIM>
__global__ void __launch_bounds__(128) walk_exact_kernel(ExactArgs E) {
    constexpr int NAX = (P_ > 0) ? (P_ + Q_) : CMFW_MAX_AXES;
    constexpr int PM = (P_ > 0) ? P_ : 8;
    constexpr int QM = (P_ > 0) ? Q_ : 7;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)E.n_traj * E.K) return;
    const int t = (int)(gid / E.K), k = (int)(gid % E.K);
    const int P = (P_ > 0) ? P_ : E.p;
    const int Q = (P_ > 0) ? Q_ : E.q;
    const int naxes = P + Q;
    const cmfw_traj_in &in = E.in[t];
    int si = 0, sj = 1, sc = DIM - 1;
    if (E.pairs) {
        const int sel = E.pairs[t];
        if (sel >= 0) {
            si = min((sel >> 8) & 15, DIM - 1);
            sj = min((sel >> 4) & 15, DIM - 1);
            sc = min(sel & 15, DIM - 1);
        }
    }

    Mod M;
    {
        const uint32_t m = E.primes[k];
        M.m = m;
        uint32_t inv = 1;
        for (int i = 0; i < 5; ++i) inv *= 2u - m * inv;
        M.ninv = 0u - inv;
        const uint64_t r1 = (((uint64_t)1) << 32) % m;
        M.r1 = (uint32_t)r1;
        M.r2 = (uint32_t)((r1 * r1) % m);
    }
    uint8_t ok = 1;
    int absd[NAX];
    uint32_t neg;
    const int maxabs = load_direction<NAX>(in, naxes, absd, neg);
    if (maxabs < 0 || E.N <= 0 || E.h <= 0 || E.N - 2 * E.h <= 0) ok = 0;

    // Positions as residues; start coordinates must be integers.
    uint32_t pr[NAX];
    const uint32_t one = M.r1;
#pragma unroll
    for (int a = 0; a < NAX; ++a) {
        double v = (a < naxes) ? in.start[a] : 0.0;
        if (v != floor(v) || fabs(v) >= 9.0e15) { ok = 0; v = 0.0; }
        pr[a] = mont_from_i64((long long)v, M);
    }
    const uint32_t zn = mont_from_i64(E.zn, M), zd = mont_from_i64(E.zd, M);

    uint32_t m[DIM][DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i)
#pragma unroll
        for (int j = 0; j < DIM; ++j) m[i][j] = (i == j) ? one : 0u;
    const int cp1 = E.N - 2 * E.h, cp2 = E.N - E.h;
    uint32_t *out = E.res + (size_t)t * 6 * E.K;

    for (int step = 1; step <= E.N && ok; ++step) {
        for (int level = maxabs; level >= 1 && ok; --level) {
            uint32_t mask = level_mask<NAX>(absd, level);
            while (mask) {
                const int axis = top_axis(mask);
                mask &= ~(1u << axis);
                const bool up = !((neg >> axis) & 1u);
                const bool is_x = axis < P;
                const bool inverse = is_x ? !up : up;
                uint32_t pa = 0;
#pragma unroll
                for (int a = 0; a < NAX; ++a) pa = (a == axis) ? pr[a] : pa;
                const uint32_t a_res = up ? pa : msub(pa, one, M);  // axis denominator
                // eval shift: -1 for x-, +1 for y+
                uint32_t xv[PM], yv[QM > 0 ? QM : 1];
#pragma unroll
                for (int j = 0; j < PM; ++j) {
                    uint32_t v = (j < P) ? pr[j] : 0u;
                    if (j == axis && inverse) v = msub(v, one, M);
                    xv[j] = v;
                }
#pragma unroll
                for (int i = 0; i < QM; ++i) {
                    uint32_t v = (i < Q) ? msub(pr[P + i], one, M) : 0u;
                    if (P + i == axis && inverse) v = madd(v, one, M);
                    yv[i] = v;
                }
                // prod(theta + v) coefficients mod the prime
                uint32_t px[PM + 1], py[(QM > 0 ? QM : 0) + 1];
                px[0] = one;
#pragma unroll
                for (int c = 1; c <= PM; ++c) px[c] = 0u;
#pragma unroll
                for (int j = 0; j < PM; ++j)
                    if (j < P) {
#pragma unroll
                        for (int c = j + 1; c >= 1; --c) px[c] = madd(mmul(px[c], xv[j], M), px[c - 1], M);
                        px[0] = mmul(px[0], xv[j], M);
                    }
                py[0] = one;
#pragma unroll
                for (int c = 1; c <= QM; ++c) py[c] = 0u;
#pragma unroll
                for (int i = 0; i < QM; ++i)
                    if (i < Q) {
#pragma unroll
                        for (int c = i + 1; c >= 1; --c) py[c] = madd(mmul(py[c], yv[i], M), py[c - 1], M);
                        py[0] = mmul(py[0], yv[i], M);
                    }
                // zd * D(theta): zd*theta*prod(theta + y - 1) - zn*prod(theta + x)
                uint32_t d[DIM + 1];
#pragma unroll
                for (int c = 0; c <= DIM; ++c) {
                    uint32_t v = (c <= PM && c <= P) ? msub(0u, mmul(zn, px[c <= PM ? c : 0], M), M) : 0u;
                    if (c >= 1 && c - 1 <= QM && c - 1 <= Q) v = madd(v, mmul(zd, py[(c - 1) <= QM ? (c - 1) : 0], M), M);
                    d[c] = v;
                }
                const uint32_t lead = d[DIM];
                const uint32_t al_ = mmul(a_res, lead, M);
                if (al_ == 0u) { ok = 0; break; }
                const uint32_t inv_al = minv_fermat(al_, M);
                const uint32_t inva = mmul(inv_al, lead, M);   // 1/a
                const uint32_t il = mmul(inv_al, a_res, M);    // 1/lead
                uint32_t col[DIM];
#pragma unroll
                for (int i = 0; i < DIM; ++i) col[i] = msub(0u, mmul(d[i], il, M), M);
                if (!inverse) {
#pragma unroll
                    for (int r = 0; r < DIM; ++r) {
                        uint32_t dot = 0;
#pragma unroll
                        for (int i = 0; i < DIM; ++i) dot = madd(dot, mmul(m[r][i], col[i], M), M);
#pragma unroll
                        for (int j = 0; j < DIM - 1; ++j) m[r][j] = madd(m[r][j], mmul(m[r][j + 1], inva, M), M);
                        m[r][DIM - 1] = madd(m[r][DIM - 1], mmul(dot, inva, M), M);
                    }
                } else {
                    uint32_t be[DIM];
                    be[DIM - 1] = one;
#pragma unroll
                    for (int j = DIM - 2; j >= 0; --j) be[j] = msub(0u, mmul(be[j + 1], inva, M), M);
                    uint32_t db = 0;
#pragma unroll
                    for (int i = 0; i < DIM; ++i) db = madd(db, mmul(be[i], col[i], M), M);
                    const uint32_t sd = madd(one, mmul(db, inva, M), M);
                    if (sd == 0u) { ok = 0; break; }
                    const uint32_t isd = minv_fermat(sd, M);
#pragma unroll
                    for (int r = 0; r < DIM; ++r) {
                        uint32_t al[DIM];
                        al[DIM - 1] = 0u;
#pragma unroll
                        for (int j = DIM - 2; j >= 0; --j) al[j] = msub(m[r][j], mmul(al[j + 1], inva, M), M);
                        uint32_t da = 0;
#pragma unroll
                        for (int i = 0; i < DIM; ++i) da = madd(da, mmul(al[i], col[i], M), M);
                        const uint32_t tt = mmul(msub(m[r][DIM - 1], mmul(da, inva, M), M), isd, M);
#pragma unroll
                        for (int j = 0; j < DIM; ++j) m[r][j] = madd(al[j], mmul(be[j], tt, M), M);
                    }
                }
#pragma unroll
                for (int a = 0; a < NAX; ++a)
                    if (a == axis) pr[a] = up ? madd(pr[a], one, M) : msub(pr[a], one, M);
            }
        }
        if (!ok) break;
        const int s = (step == cp1) ? 0 : (step == cp2) ? 1 : (step == E.N) ? 2 : -1;
        if (s >= 0) {
            uint32_t vi = 0, vj = 0;
#pragma unroll
            for (int r = 0; r < DIM; ++r)
#pragma unroll
                for (int c = 0; c < DIM; ++c) {
                    vi = (r == si && c == sc) ? m[r][c] : vi;
                    vj = (r == sj && c == sc) ? m[r][c] : vj;
                }
            out[(s * 2 + 0) * E.K + k] = mfrom(vi, M);
            out[(s * 2 + 1) * E.K + k] = mfrom(vj, M);
        }
    }
    E.prime_ok[(size_t)t * E.K + k] = ok;
}

typedef void (*exact_kernel_t)(ExactArgs);

static exact_kernel_t pick_exact(int p, int q, int dim) {
#define CMFW_CASE(P, Q, D) if (p == P && q == Q && dim == D) return walk_exact_kernel<P, Q, D>;
    CMFW_FAMILY_CASES
#undef CMFW_CASE
    switch (dim) {
        case 2: return walk_exact_kernel<0, 0, 2>;
        case 3: return walk_exact_kernel<0, 0, 3>;
        case 4: return walk_exact_kernel<0, 0, 4>;
        case 5: return walk_exact_kernel<0, 0, 5>;
        case 6: return walk_exact_kernel<0, 0, 6>;
        case 7: return walk_exact_kernel<0, 0, 7>;
        case 8: return walk_exact_kernel<0, 0, 8>;
    }
    return nullptr;
}

cudaError_t launch_walk_exact(const cmfw_traj_in *in, int n_traj, int p, int q, int dim, int N, int h,
                              long long zn, long long zd, const uint32_t *primes, int K, const int *pairs,
                              uint32_t *res, uint8_t *prime_ok, cudaStream_t s) {
    ExactArgs E;
    E.in = in;
    E.primes = primes;
    E.res = res;
    E.prime_ok = prime_ok;
    E.pairs = pairs;
    E.n_traj = n_traj;
    E.N = N;
    E.h = h;
    E.K = K;
    E.p = p;
    E.q = q;
    E.dim = dim;
    E.zn = zn;
    E.zd = zd;
    exact_kernel_t k = pick_exact(p, q, dim);
    if (!k) return cudaErrorInvalidValue;
    const long long threads = (long long)n_traj * K;
    const int block = 128;
    k<<<(unsigned)((threads + block - 1) / block), block, 0, s>>>(E);
    return cudaGetLastError();
}

}  // namespace cmfw
