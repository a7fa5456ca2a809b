// Exact ratios from the exact walk's residues, on the device.
//
// The exact walk (walk_exact_kernel) leaves, per trajectory and snapshot
// depth, the residues a_k, b_k of two entries of one column of the walk
// matrix modulo K primes. Their ratio is a rational number n / d; here one
// warp recovers it:
//
//   1. u_k = a_k / b_k mod p_k for every usable prime (ok and b_k != 0),
//      one prime per lane (lane-strided), Montgomery arithmetic;
//   2. Garner's mixed-radix Chinese remaindering over the first F = U - 4
//      usable primes: digits v_j with X = sum_j v_j p_0 ... p_{j-1} = u_k
//      mod every p_k, X < P = p_0 ... p_{F-1}. Lanes hold the primes, the
//      digit of step j is computed by its prime's lane and broadcast, and
//      every later prime's running sum is advanced in parallel;
//   3. X and P as multi-precision integers (32-bit words in shared memory,
//      Horner over the digits);
//   4. rational reconstruction: the half-extended Euclidean algorithm on
//      (P, X) stops at the first remainder r below 2^Lb <= sqrt(P / 2)
//      (Wang's bound); then r = t X mod P, so X = r / t, and the fraction
//      is accepted when 2 * 2^Lb * |t| < P -- the bound under which it is
//      the unique one (P. S. Wang, 1981; Collins and Encarnacion, 1994);
//   5. the result is checked against the 4 held-out primes: n b_h = a_h d
//      modulo each.
//
// Multi-precision steps are whole-warp operations over 32-word chunks:
// a word product's high half moves one lane up by shuffle, and the carry
// (or borrow) chain of a chunk is resolved at once from two ballots: with
// g = "this word generates a carry" and p = "this word passes one on"
// (never both), the carries into the words are the sum bits of
// (g | p) + g + carry_in xor p, the carry out its bit 32. Quotients of
// the Euclidean steps are taken from the leading bits of both operands and
// never exceed the true quotient, so every remainder stays non-negative; a
// step with a large quotient is done as several such partial steps.
//
// Every loop is bounded; a task that would exceed its bound reports
// "undetermined" and the caller adds primes. Status per task: 0 = the
// fraction, 1 = the denominator vanishes modulo every usable prime (an
// exact zero), 2 = undetermined (too few primes, bound not met, or a
// held-out prime disagrees), 3 = no prime usable (the exact walk is
// singular).
#include <cstdio>

#include "cmfw.h"
#include "cmfw_internal.cuh"

namespace cmfw {
cmfw_status record_error(cmfw_status s, const char *msg);

namespace {

constexpr unsigned FULL = 0xffffffffu;

struct ReconArgs {
    const uint32_t *res;    // [n][3][2][stride]
    const uint8_t *ok;      // [n][stride]
    const uint32_t *primes; // [K], each in (2^30, 2^31)
    int n_tasks, stride, K, W;
    uint32_t *num, *den;    // [n_tasks][W] little-endian words
    int *num_len, *den_len; // words used
    int8_t *sign;           // of the numerator
    uint8_t *status;
};

__device__ __forceinline__ Mod make_mod(uint32_t m) {
    Mod M;
    M.m = m;
    uint32_t inv = 1;
    for (int i = 0; i < 5; ++i) inv *= 2u - m * inv;
    M.ninv = 0u - inv;
    const uint64_t r1 = (((uint64_t)1) << 32) % m;
    M.r1 = (uint32_t)r1;
    M.r2 = (uint32_t)((r1 * r1) % m);
    return M;
}

// x mod m for x < 2^31 < 2 m (every prime is above 2^30)
__device__ __forceinline__ uint32_t red2(uint32_t x, uint32_t m) { return x >= m ? x - m : x; }

// carries into the 32 words of a chunk and out of it (see the file comment)
__device__ __forceinline__ uint32_t chain(bool g, bool p, uint32_t cin, uint32_t *cout) {
    const uint32_t G = __ballot_sync(FULL, g), P = __ballot_sync(FULL, p);
    const uint64_t s = (uint64_t)(G | P) + (uint64_t)G + (uint64_t)cin;
    *cout = (uint32_t)(s >> 32);
    return (uint32_t)s ^ P;
}

__device__ __forceinline__ int trim(const uint32_t *B, int len) {
    while (len > 0 && B[len - 1] == 0u) --len;
    return len;
}

__device__ __forceinline__ int bitlen(const uint32_t *B, int len) {
    return len == 0 ? 0 : 32 * (len - 1) + (32 - __clz(B[len - 1]));
}

// bits [e, e + 64) of B (zero above its length)
__device__ __forceinline__ uint64_t bits64(const uint32_t *B, int len, int e) {
    const int w = e >> 5, b = e & 31;
    auto word = [&](int i) -> uint64_t { return (i >= 0 && i < len) ? (uint64_t)B[i] : 0ull; };
    const uint64_t lo = word(w) | (word(w + 1) << 32);
    const uint64_t hi = word(w + 2);
    return b == 0 ? lo : ((lo >> b) | (hi << (64 - b)));
}

// word i of (B << sh)
__device__ __forceinline__ uint32_t shifted_word(const uint32_t *B, int len, int ws, int bs, int i) {
    const int j = i - ws;
    const uint32_t a = (j >= 0 && j < len) ? B[j] : 0u;
    if (bs == 0) return a;
    const uint32_t c = (j - 1 >= 0 && j - 1 < len) ? B[j - 1] : 0u;
    return (a << bs) | (c >> (32 - bs));
}

// B = B * m + a; returns the new length (at most len + 1)
__device__ int mul_small_add(uint32_t *B, int len, uint32_t m, uint32_t a) {
    const int lane = threadIdx.x & 31;
    const int nl = len + 1;
    uint32_t hi_in = a, cin = 0;
    for (int c0 = 0; c0 < nl; c0 += 32) {
        const int i = c0 + lane;
        const uint64_t x = (i < len) ? (uint64_t)B[i] * m : 0ull;
        const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
        uint32_t hp = __shfl_up_sync(FULL, hi, 1);
        if (lane == 0) hp = hi_in;
        const uint64_t y = (uint64_t)lo + hp;
        const bool g = (y >> 32) != 0, p = !g && (uint32_t)y == 0xffffffffu;
        uint32_t cout;
        const uint32_t C = chain(g, p, cin, &cout);
        if (i < nl) B[i] = (uint32_t)y + ((C >> lane) & 1u);
        hi_in = __shfl_sync(FULL, hi, 31);
        cin = cout;
        __syncwarp();
    }
    return trim(B, nl);
}

// R = R - q (S << sh) when the result is known to be non-negative
__device__ int sub_mul_shift(uint32_t *R, int lenR, const uint32_t *S, int lenS, uint32_t q, int sh) {
    const int lane = threadIdx.x & 31;
    const int ws = sh >> 5, bs = sh & 31;
    uint32_t hi_in = 0, c_mul = 0, b_sub = 0;
    for (int c0 = 0; c0 < lenR; c0 += 32) {
        const int i = c0 + lane;
        const uint64_t x = (uint64_t)shifted_word(S, lenS, ws, bs, i) * q;
        const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
        uint32_t hp = __shfl_up_sync(FULL, hi, 1);
        if (lane == 0) hp = hi_in;
        const uint64_t y = (uint64_t)lo + hp;
        const bool g = (y >> 32) != 0, p = !g && (uint32_t)y == 0xffffffffu;
        uint32_t cout;
        const uint32_t C = chain(g, p, c_mul, &cout);
        const uint32_t Y = (uint32_t)y + ((C >> lane) & 1u);  // word i of q (S << sh)
        const uint32_t r = (i < lenR) ? R[i] : 0u;
        uint32_t bout;
        const uint32_t B = chain(r < Y, r == Y, b_sub, &bout);
        if (i < lenR) R[i] = r - Y - ((B >> lane) & 1u);
        hi_in = __shfl_sync(FULL, hi, 31);
        c_mul = cout;
        b_sub = bout;
        __syncwarp();
    }
    return trim(R, lenR);
}

// T = T + q (S << sh); cap = words available; returns the new length
__device__ int add_mul_shift(uint32_t *T, int lenT, const uint32_t *S, int lenS, uint32_t q, int sh, int cap) {
    const int lane = threadIdx.x & 31;
    const int ws = sh >> 5, bs = sh & 31;
    int nl = max(lenT, lenS + ws + 1) + 1;
    if (nl > cap) nl = cap;
    uint32_t hi_in = 0, c_mul = 0, c_add = 0;
    for (int c0 = 0; c0 < nl; c0 += 32) {
        const int i = c0 + lane;
        const uint64_t x = (uint64_t)shifted_word(S, lenS, ws, bs, i) * q;
        const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
        uint32_t hp = __shfl_up_sync(FULL, hi, 1);
        if (lane == 0) hp = hi_in;
        const uint64_t y = (uint64_t)lo + hp;
        const bool g = (y >> 32) != 0, p = !g && (uint32_t)y == 0xffffffffu;
        uint32_t cout;
        const uint32_t C = chain(g, p, c_mul, &cout);
        const uint32_t Y = (uint32_t)y + ((C >> lane) & 1u);
        const uint32_t t = (i < lenT) ? T[i] : 0u;
        const uint64_t z = (uint64_t)t + Y;
        const bool g2 = (z >> 32) != 0, p2 = !g2 && (uint32_t)z == 0xffffffffu;
        uint32_t aout;
        const uint32_t A = chain(g2, p2, c_add, &aout);
        if (i < nl) T[i] = (uint32_t)z + ((A >> lane) & 1u);
        hi_in = __shfl_sync(FULL, hi, 31);
        c_mul = cout;
        c_add = aout;
        __syncwarp();
    }
    return trim(T, nl);
}

// -1, 0, 1 as A <, =, > B
__device__ int compare(const uint32_t *A, int la, const uint32_t *B, int lb) {
    if (la != lb) return la < lb ? -1 : 1;
    for (int i = la - 1; i >= 0; --i)
        if (A[i] != B[i]) return A[i] < B[i] ? -1 : 1;
    return 0;
}

// B mod m (m odd, below 2^31): each lane sums its words times (2^32)^i
__device__ uint32_t mod_small(const uint32_t *B, int len, uint32_t m) {
    const int lane = threadIdx.x & 31;
    const Mod M = make_mod(m);
    // Montgomery forms of 2^32 (= R) and of R^32
    const uint32_t R = M.r2;  // mto(2^32 mod m) = R^2 mod m
    uint32_t R32 = R;
    for (int k = 0; k < 5; ++k) R32 = mmul(R32, R32, M);  // R^32
    uint32_t pw = M.r1;                                   // R^lane
    for (int k = 0; k < lane; ++k) pw = mmul(pw, R, M);
    uint32_t acc = 0;
    for (int i = lane; i < len; i += 32) {
        acc = madd(acc, mmul(mto(B[i] % m, M), pw, M), M);
        pw = mmul(pw, R32, M);
    }
    for (int o = 16; o > 0; o >>= 1) acc = madd(acc, __shfl_xor_sync(FULL, acc, o), M);
    return mfrom(acc, M);
}

__global__ void __launch_bounds__(32) exact_reconstruct_kernel(ReconArgs A) {
    extern __shared__ __align__(16) uint32_t sm[];
    const int task = blockIdx.x;
    if (task >= A.n_tasks) return;
    const int lane = threadIdx.x;
    const int K = A.K, W = A.W;
    uint32_t *up = sm;           // usable primes, compacted [K]
    uint32_t *uu = up + K;       // their ratio residues u (plain) [K]
    uint32_t *acc = uu + K;      // Garner running sums (Montgomery) [K]
    uint32_t *prd = acc + K;     // running products of earlier primes (Montgomery) [K]
    uint32_t *ha = prd + K;      // held-out a, b (plain) [8]
    uint32_t *R0 = ha + 8, *R1 = R0 + W, *T0 = R1 + W, *T1 = T0 + W;
    const int t = task / 3, s = task % 3;
    const uint32_t *ra = A.res + ((size_t)t * 3 + s) * 2 * A.stride;
    const uint32_t *rb = ra + A.stride;
    const uint8_t *ok = A.ok + (size_t)t * A.stride;

    // 1. usable primes in order, with u = a / b
    int U = 0;
    bool any_ok = false, bad_prime = false;
    for (int k0 = 0; k0 < K; k0 += 32) {
        const int k = k0 + lane;
        const bool o = k < K && ok[k];
        if (k < K) {
            const uint32_t p = A.primes[k];
            bad_prime |= p <= (1u << 30) || p >= (1u << 31) || !(p & 1u);
        }
        const uint32_t b = o ? rb[k] : 0u;
        const bool use = o && b != 0u;
        any_ok |= __any_sync(FULL, o);
        const uint32_t bal = __ballot_sync(FULL, use);
        if (use) {
            const int at = U + __popc(bal & ((1u << lane) - 1u));
            const uint32_t p = A.primes[k];
            const Mod M = make_mod(p);
            const uint32_t a = ra[k] % p;
            const uint32_t u = mfrom(mmul(mto(a, M), minv_fermat(mto(b % p, M), M), M), M);
            up[at] = p;
            uu[at] = u;
        }
        U += __popc(bal);
    }
    __syncwarp();
    bad_prime = __any_sync(FULL, bad_prime);
    uint8_t st = 2;
    int8_t sg = 1;
    int ln = 0, ld = 0;
    if (bad_prime) {
        st = 2;  // outside the arithmetic's range: never a wrong value
    } else if (!any_ok) {
        st = 3;
    } else if (U == 0) {
        st = 1;
    } else if (U >= 6) {
        const int F = U - 4;
        // the held-out primes' a and b: find them again (the last 4 usable)
        if (lane == 0) {
            int seen = 0;
            for (int k = K - 1; k >= 0 && seen < 4; --k)
                if (ok[k] && rb[k] != 0u) {
                    ha[2 * (3 - seen)] = ra[k];
                    ha[2 * (3 - seen) + 1] = rb[k];
                    ++seen;
                }
        }
        // 2. Garner: acc_i = sum_{m<j} v_m P_m mod p_i, prd_i = P_j mod p_i
        for (int i = lane; i < F; i += 32) {
            const Mod M = make_mod(up[i]);
            acc[i] = 0u;
            prd[i] = M.r1;
        }
        __syncwarp();
        // the digit v_j replaces u_j in uu (only step j reads u_j)
        for (int j = 0; j < F; ++j) {
            uint32_t v = 0;
            if ((j & 31) == lane) {
                const Mod M = make_mod(up[j]);
                const uint32_t d = msub(mto(uu[j], M), acc[j], M);
                v = mfrom(mmul(d, minv_fermat(prd[j], M), M), M);
                uu[j] = v;
            }
            v = __shfl_sync(FULL, v, j & 31);
            const uint32_t pj = up[j];
            for (int i = j + 1 + ((lane - (j + 1)) & 31); i < F; i += 32) {
                const Mod M = make_mod(up[i]);
                acc[i] = madd(acc[i], mmul(mto(red2(v, up[i]), M), prd[i], M), M);
                prd[i] = mmul(prd[i], mto(red2(pj, up[i]), M), M);
            }
            __syncwarp();
        }
        // 3. X (Horner over the digits) into T0, P into R0
        if (lane == 0) {
            T0[0] = 0u;
            R0[0] = 1u;
        }
        __syncwarp();
        int lx = 0, lp = 1;
        for (int j = F - 1; j >= 0; --j) lx = mul_small_add(T0, lx, up[j], uu[j]);  // X = X p_j + v_j
        for (int j = 0; j < F; ++j) lp = mul_small_add(R0, lp, up[j], 0u);
        // 4. half-extended Euclid on (P, X): R0 = P, R1 = X, T0 = 0, T1 = 1
        //    (X moves from T0 to R1; magnitudes of t, whose signs alternate)
        for (int i = lane; i < W; i += 32) R1[i] = i < lx ? T0[i] : 0u;
        __syncwarp();
        int l0 = lp, l1 = trim(R1, lx);
        for (int i = lane; i < W; i += 32) {
            T0[i] = 0u;
            T1[i] = i == 0 ? 1u : 0u;
        }
        __syncwarp();
        int lt0 = 0, lt1 = 1;
        bool neg1 = false;  // sign of t1 (t0 has the other)
        const int bits_p = bitlen(R0, l0);
        const int Lb = (bits_p - 2) / 2;
        long long budget = 4ll * 32 * W + 4096;
        bool done = false;
        while (!done && budget > 0) {
            if (bitlen(R1, l1) <= Lb) {
                done = true;
                break;
            }
            // partial steps until R0 < R1
            while (budget-- > 0) {
                const int c = compare(R0, l0, R1, l1);
                if (c < 0) break;
                const int b0 = bitlen(R0, l0), b1 = bitlen(R1, l1);
                const int e0 = b0 > 64 ? b0 - 64 : 0, e1 = b1 > 32 ? b1 - 32 : 0;
                const uint64_t a64 = bits64(R0, l0, e0);
                const uint64_t d64 = (bits64(R1, l1, e1) & 0xffffffffull) + 1ull;
                uint64_t Q = a64 / d64;
                int sh = e0 - e1;
                if (sh < 0) {
                    Q = (-sh >= 64) ? 0ull : (Q >> (-sh));
                    sh = 0;
                }
                if (Q > 0xffffffffull) Q = 0xffffffffull;
                if (Q == 0) {
                    Q = 1;  // R0 >= R1 (compared above): one R1 fits
                    sh = 0;
                }
                l0 = sub_mul_shift(R0, l0, R1, l1, (uint32_t)Q, sh);
                lt0 = add_mul_shift(T0, lt0, T1, lt1, (uint32_t)Q, sh, W);
            }
            // swap the roles: (R0, R1) = (R1, R0), (T0, T1) = (T1, T0)
            uint32_t *tmp = R0; R0 = R1; R1 = tmp;
            int ti = l0; l0 = l1; l1 = ti;
            tmp = T0; T0 = T1; T1 = tmp;
            ti = lt0; lt0 = lt1; lt1 = ti;
            neg1 = !neg1;
        }
        // 5. accept: bound on |t|, then the held-out primes
        const int bt = bitlen(T1, lt1);
        if (done && lt1 > 0 && bt + Lb + 1 <= bits_p - 1) {
            bool good = true;
            for (int h = 0; h < 4 && good; ++h) {
                const uint32_t a = ha[2 * h], b = ha[2 * h + 1];
                // the held-out prime of slot h is the (U - 4 + h)-th usable
                const uint32_t p = up[F + h];
                const Mod M = make_mod(p);
                const uint32_t nm = mod_small(R1, l1, p), dm = mod_small(T1, lt1, p);
                // n b = a d (mod p), with n = -R1 when t1 < 0
                uint32_t lhs = mmul(mto(nm, M), mto(b % p, M), M);
                if (neg1) lhs = msub(0u, lhs, M);
                const uint32_t rhs = mmul(mto(a % p, M), mto(dm, M), M);
                good = lhs == rhs;
            }
            if (good) {
                st = 0;
                sg = (neg1 && l1 > 0) ? -1 : 1;
                ln = l1;
                ld = lt1;
                uint32_t *on = A.num + (size_t)task * W, *od = A.den + (size_t)task * W;
                for (int i = lane; i < W; i += 32) {
                    on[i] = i < l1 ? R1[i] : 0u;
                    od[i] = i < lt1 ? T1[i] : 0u;
                }
            }
        }
    }
    if (lane == 0) {
        A.status[task] = st;
        A.sign[task] = sg;
        A.num_len[task] = ln;
        A.den_len[task] = ld;
    }
}

}  // namespace

size_t exact_recon_smem(int K) {
    return ((size_t)4 * K + 8 + 4 * (size_t)cmfw_exact_recon_words(K)) * sizeof(uint32_t);
}

static cudaError_t launch_exact_reconstruct(const uint32_t *res, const uint8_t *ok, const uint32_t *primes, int n_traj,
                                     int stride, int K, uint32_t *num, uint32_t *den, int *num_len, int *den_len,
                                     int8_t *sign, uint8_t *status, cudaStream_t s) {
    ReconArgs A;
    A.res = res;
    A.ok = ok;
    A.primes = primes;
    A.n_tasks = 3 * n_traj;
    A.stride = stride;
    A.K = K;
    A.W = cmfw_exact_recon_words(K);
    A.num = num;
    A.den = den;
    A.num_len = num_len;
    A.den_len = den_len;
    A.sign = sign;
    A.status = status;
    const size_t shm = exact_recon_smem(K);
    cudaError_t e = cudaFuncSetAttribute((const void *)exact_reconstruct_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return e;
    exact_reconstruct_kernel<<<A.n_tasks, 32, shm, s>>>(A);
    return cudaGetLastError();
}

}  // namespace cmfw

using namespace cmfw;

extern "C" int cmfw_exact_recon_words(int K) { return K < 1 ? 0 : (31 * K + 31) / 32 + 4; }

extern "C" cmfw_status cmfw_exact_reconstruct(const uint32_t *d_res, const uint8_t *d_prime_ok,
                                              const uint32_t *d_primes, int n_traj, int stride, int K,
                                              uint32_t *d_num, uint32_t *d_den, int *d_num_words,
                                              int *d_den_words, int8_t *d_sign, uint8_t *d_status, void *stream) {
    if (n_traj < 0 || K < 1 || K > stride || stride > CMFW_MAX_EXACT_PRIMES)
        return record_error(CMFW_EINVAL, "exact reconstruction: need 1 <= K <= stride <= 4096 and n_traj >= 0");
    if (n_traj == 0) return CMFW_OK;
    if (!d_res || !d_prime_ok || !d_primes || !d_num || !d_den || !d_num_words || !d_den_words || !d_sign ||
        !d_status)
        return record_error(CMFW_EINVAL, "exact reconstruction: NULL buffer");
    cudaError_t e = launch_exact_reconstruct(d_res, d_prime_ok, d_primes, n_traj, stride, K, d_num, d_den,
                                             d_num_words, d_den_words, d_sign, d_status, (cudaStream_t)stream);
    if (e != cudaSuccess) return record_error(CMFW_ECUDA, cudaGetErrorString(e));
    return CMFW_OK;
}
