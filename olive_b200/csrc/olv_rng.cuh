// Counter-based random draws for the synthetic workloads.  The mixing
// function is the SplitMix64 output function (Steele, Lea, Flood 2014)
// applied to seed + counter * golden ratio; every draw is a pure function of
// (seed, counter), so the GPU and a CPU restatement generate identical graphs.
#pragma once
#include <stdint.h>

namespace olv {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t hash64(uint64_t seed, uint64_t ctr) {
    return mix64(seed + ctr * 0x9E3779B97F4A7C15ULL);
}

// Seeded bijection on [0, 2^bits): three rounds of add, odd multiply and
// xor-shift, each invertible modulo 2^bits.
__host__ __device__ __forceinline__ uint32_t permute_bits(uint32_t x, int bits, uint64_t seed) {
    const uint64_t mask = (bits >= 64) ? ~0ULL : ((1ULL << bits) - 1);
    int sh = (bits + 1) / 2;
    if (sh < 1) sh = 1;
    uint64_t y = x;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const uint64_t m = hash64(seed, 2 * r) | 1ULL;
        const uint64_t c = hash64(seed, 2 * r + 1);
        y = (y + c) & mask;
        y = (y * m) & mask;
        y ^= (y >> sh);
        y &= mask;
    }
    return (uint32_t)y;
}

// RMAT quadrant thresholds on a 32-bit draw for (a,b,c,d) = (.57,.19,.19,.05).
constexpr uint32_t kRmatA = 2448131359u;    // round(0.57 * 2^32)
constexpr uint32_t kRmatAB = 3264175145u;   // round(0.76 * 2^32)
constexpr uint32_t kRmatABC = 4080218931u;  // round(0.95 * 2^32)

__host__ __device__ __forceinline__ void rmat_edge(int scale, uint64_t seed, uint64_t i,
                                                   uint32_t *src, uint32_t *dst) {
    uint32_t s = 0, d = 0;
    for (int b = 0; b < scale; b++) {
        const uint32_t u = (uint32_t)(hash64(seed, i * 64 + (uint64_t)b) >> 32);
        const uint32_t sb = u >= kRmatAB;
        const uint32_t db = (u >= kRmatA && u < kRmatAB) || u >= kRmatABC;
        s = (s << 1) | sb;
        d = (d << 1) | db;
    }
    *src = s;
    *dst = d;
}

}  // namespace olv
