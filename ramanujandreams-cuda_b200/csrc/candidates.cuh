// The seeded candidate generator of the delta search: direction component a
// of candidate idx is lo + (a 16-bit field of a splitmix64 draw) mod
// (hi - lo + 1), one 64-bit draw per four components. Counter-based, so any
// candidate is drawn on its own (scoring, filtering and record building
// draw the same directions without materialising them).
#pragma once

#include <cstdint>

namespace cmfw {

// splitmix64 (S. Vigna's finaliser of the SplitMix generator).
__host__ __device__ inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// The draw holding components 4w .. 4w+3 of candidate idx.
__host__ __device__ inline uint64_t candidate_draw(uint64_t seed, long long idx, int w) {
    return splitmix64(seed ^ ((uint64_t)idx * 4ull + (uint64_t)w) * 0xD1B54A32D192ED03ull);
}

// x mod d for x < 2^16 and d >= 1 without a division. With
// m = floor((2^32 - 1) / d) + 1 (ceil(2^32 / d), or 2^32 / d for d a power
// of two), x m / 2^32 = x / d + x e / 2^32 with 0 <= e < 1. For d <= 2^16,
// x e / 2^32 < 2^-16 <= 1 / d, less than the distance from x / d to the
// next integer, so floor(x m / 2^32) = floor(x / d). For d > 2^16, m <= 2^16
// and x m < 2^32: the quotient is 0 = floor(x / d).
struct SmallMod {
    uint32_t d;
    uint64_t m;
    __host__ __device__ explicit SmallMod(uint32_t d_) : d(d_), m((uint64_t)(0xFFFFFFFFu / d_) + 1ull) {}
    __host__ __device__ uint32_t operator()(uint32_t x) const { return x - (uint32_t)(((uint64_t)x * m) >> 32) * d; }
};

// Components 0..15 of candidate idx (16-bit field a & 3 of draw a >> 2,
// reduced modulo the span, plus lo); a direction of naxes axes uses the
// first naxes.
__host__ __device__ inline void candidate_direction(uint64_t seed, long long idx, int lo, const SmallMod &mod,
                                                    int comp[16]) {
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        const uint64_t d = candidate_draw(seed, idx, w);
#pragma unroll
        for (int q = 0; q < 4; ++q) comp[4 * w + q] = lo + (int)mod((uint32_t)((d >> (16 * q)) & 0xFFFFull));
    }
}

// Network features of a direction d[0..naxes) of family `family` (0..4 =
// 3F2, 4F3, 5F4, 6F5, 8F7; the first p axes are x-axes, the rest y-axes):
// how many x components have |d| = 0, 1, 2, 3 and >= 4, over p (slots
// 0..4), the same for the y components over q (5..9), the negative x and y
// components over p and q (10, 11), zeros (12..14), and the family one-hot
// (15..19). At a symmetric start (the zeta point: all x equal, all y
// equal) the walk depends on a direction mostly through these counts, and
// directions that differ only by permuting x or y components get the same
// features.
__host__ __device__ inline int family_p(int family) {
    return family == 0 ? 3 : family == 1 ? 4 : family == 2 ? 5 : family == 3 ? 6 : 8;
}
template <class GET>
__host__ __device__ inline void direction_features(GET comp, int naxes, int family, float *f /* 20 */) {
    for (int k = 0; k < 20; ++k) f[k] = 0.0f;
    int p = family_p(family);
    if (p > naxes) p = naxes;
    const int q = naxes - p;
    for (int a = 0; a < naxes && a < 15; ++a) {
        const int v = comp(a);
        const int m = v < 0 ? -v : v;
        const int bin = m < 4 ? m : 4;
        const bool x = a < p;
        f[(x ? 0 : 5) + bin] += 1.0f;
        if (v < 0) f[x ? 10 : 11] += 1.0f;
    }
    const float ip = p > 0 ? 1.0f / (float)p : 0.0f, iq = q > 0 ? 1.0f / (float)q : 0.0f;
    for (int k = 0; k < 5; ++k) {
        f[k] *= ip;
        f[5 + k] *= iq;
    }
    f[10] *= ip;
    f[11] *= iq;
    if (family >= 0 && family < 5) f[15 + family] = 1.0f;
}

}  // namespace cmfw
