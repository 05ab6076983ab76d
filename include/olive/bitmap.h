/*
 * olive_b200 source-compatible header layer: Bitmap with 64-bit words in
 * managed memory and atomic set/unset (bitmap.h:44-199).  Unused by the
 * engine; kept for callers of the reference's API.
 */
#ifndef OLIVE_BITMAP_H
#define OLIVE_BITMAP_H

#include "common.h"

class Bitmap : public Managed {
public:
    Word *words;
    size_t size;       // bits
    size_t numWords;

    explicit Bitmap(size_t n) : size(n), numWords((n + 63) / 64) {
        CUDA_CHECK(cudaMallocManaged(&words, numWords * sizeof(Word)));
        memset(words, 0, numWords * sizeof(Word));
    }
    ~Bitmap() { cudaFree(words); }

    __device__ void set(size_t i) {
        atomicOr((unsigned long long *)&words[i / 64], 1ULL << (i % 64));
    }
    __device__ void unset(size_t i) {
        atomicAnd((unsigned long long *)&words[i / 64], ~(1ULL << (i % 64)));
    }
    __host__ __device__ bool get(size_t i) const { return (words[i / 64] >> (i % 64)) & 1ULL; }
    __host__ void setHost(size_t i) { words[i / 64] |= 1ULL << (i % 64); }
    __host__ void unsetHost(size_t i) { words[i / 64] &= ~(1ULL << (i % 64)); }
    __host__ void clear() { memset(words, 0, numWords * sizeof(Word)); }

    __host__ Bitmap &operator&=(const Bitmap &o) {
        for (size_t w = 0; w < numWords; w++) words[w] &= o.words[w];
        return *this;
    }
    __host__ Bitmap &operator|=(const Bitmap &o) {
        for (size_t w = 0; w < numWords; w++) words[w] |= o.words[w];
        return *this;
    }
    __host__ Bitmap &operator^=(const Bitmap &o) {
        for (size_t w = 0; w < numWords; w++) words[w] ^= o.words[w];
        return *this;
    }
    __host__ size_t count() const {
        size_t c = 0;
        for (size_t w = 0; w < numWords; w++) c += __builtin_popcountll(words[w]);
        return c;
    }
};

#endif  // OLIVE_BITMAP_H
