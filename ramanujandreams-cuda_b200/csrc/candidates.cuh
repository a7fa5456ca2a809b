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

__host__ __device__ inline int candidate_component(uint64_t seed, long long idx, int a, int lo, int span) {
    const uint64_t w = candidate_draw(seed, idx, a >> 2);
    return lo + (int)(((w >> (16 * (a & 3))) & 0xFFFFull) % (uint64_t)span);
}

}  // namespace cmfw
