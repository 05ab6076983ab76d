/*
 * olive_b200 source-compatible header layer: Bitmap (bitmap.h:44-199), a bit
 * set of 64-bit words in managed memory with the reference's public API:
 *
 *   Bitmap(), Bitmap(int numBits)                 zero-filled, capacity rounded
 *                                                 up to whole words
 *   capacity()                                    bits held (numWords * 64)
 *   set(i) / unset(i) / get(i)                    host or device; on the
 *                                                 device set/unset are atomic
 *   operator=                                     deep copy
 *   operator& / operator| / operator^             new bitmap of the larger
 *                                                 capacity; & keeps the common
 *                                                 words only, | and ^ carry the
 *                                                 longer operand's tail
 *
 * Differences, on purpose: the reference had no copy constructor, so every
 * bitmap returned by value from &, | and ^ shared its words with a temporary
 * that freed them (a double cudaFree), and its operator= replaced managed
 * words with new[] memory that the destructor then passed to cudaFree.  Here
 * copies own their words (managed memory throughout) and moves transfer them.
 * count() and clear() are additions.  Host access to the words after a kernel
 * wrote them needs a device synchronisation, as with any managed memory.
 */
#ifndef OLIVE_BITMAP_H
#define OLIVE_BITMAP_H

#include <algorithm>
#include <cstring>

#include "common.h"

class Bitmap : public Managed {
private:
    Word *words;
    int numWords;

    void allocWords(int n) {
        numWords = n;
        words = NULL;
        if (n > 0) {
            CUDA_CHECK(cudaMallocManaged(&words, (size_t)n * sizeof(Word)));
            memset(words, 0, (size_t)n * sizeof(Word));
        }
    }
    void freeWords() {
        if (words) cudaFree(words);
        words = NULL;
        numWords = 0;
    }

public:
    Bitmap() : words(NULL), numWords(0) {}

    /** Zero-filled bitmap of at least numBits bits in managed memory. */
    explicit Bitmap(int numBits) { allocWords(numBits > 0 ? ((numBits - 1) >> 6) + 1 : 0); }

    Bitmap(const Bitmap &other) {
        allocWords(other.numWords);
        if (numWords) memcpy(words, other.words, (size_t)numWords * sizeof(Word));
    }

    Bitmap(Bitmap &&other) noexcept : words(other.words), numWords(other.numWords) {
        other.words = NULL;
        other.numWords = 0;
    }

    ~Bitmap() { freeWords(); }

    /** Deep copy (bitmap.h:126-134). */
    Bitmap &operator=(const Bitmap &other) {
        if (this == &other) return *this;
        freeWords();
        allocWords(other.numWords);
        if (numWords) memcpy(words, other.words, (size_t)numWords * sizeof(Word));
        return *this;
    }

    Bitmap &operator=(Bitmap &&other) noexcept {
        if (this != &other) {
            freeWords();
            words = other.words;
            numWords = other.numWords;
            other.words = NULL;
            other.numWords = 0;
        }
        return *this;
    }

    /** Number of bits held (bitmap.h:66-69). */
    inline __host__ __device__ int capacity(void) const { return numWords << 6; }

    /** Set bit `index`; atomic on the device (bitmap.h:71-86). */
    inline __host__ __device__ void set(int index) {
        const Word bitmask = static_cast<Word>(1) << (index & 0x3f);
#ifdef __CUDA_ARCH__
        atomicOr(reinterpret_cast<unsigned long long *>(&words[index >> 6]),
                 static_cast<unsigned long long>(bitmask));
#else
        words[index >> 6] |= bitmask;
#endif
    }

    /** Clear bit `index`; atomic on the device (bitmap.h:88-103). */
    inline __host__ __device__ void unset(int index) {
        const Word bitmask = static_cast<Word>(1) << (index & 0x3f);
#ifdef __CUDA_ARCH__
        atomicAnd(reinterpret_cast<unsigned long long *>(&words[index >> 6]),
                  static_cast<unsigned long long>(~bitmask));
#else
        words[index >> 6] &= ~bitmask;
#endif
    }

    /** Bit `index` (bitmap.h:105-110). */
    inline __host__ __device__ bool get(int index) const {
        return (words[index >> 6] >> (index & 0x3f)) & 1;
    }

    /** Common words ANDed; the result has the larger capacity (bitmap.h:143-152). */
    Bitmap operator&(const Bitmap &other) const {
        Bitmap r(std::max(capacity(), other.capacity()));
        const int n = std::min(numWords, other.numWords);
        for (int i = 0; i < n; i++) r.words[i] = words[i] & other.words[i];
        return r;
    }

    /** Common words ORed, the longer operand's tail copied (bitmap.h:160-176). */
    Bitmap operator|(const Bitmap &other) const { return combine(other, false); }

    /** Common words XORed, the longer operand's tail copied (bitmap.h:184-199). */
    Bitmap operator^(const Bitmap &other) const { return combine(other, true); }

    /** Number of set bits (addition). */
    size_t count() const {
        size_t c = 0;
        for (int i = 0; i < numWords; i++) c += (size_t)__builtin_popcountll(words[i]);
        return c;
    }

    /** Clear every bit (addition). */
    void clear() {
        if (numWords) memset(words, 0, (size_t)numWords * sizeof(Word));
    }

private:
    Bitmap combine(const Bitmap &other, bool exclusive) const {
        Bitmap r(std::max(capacity(), other.capacity()));
        const int n = std::min(numWords, other.numWords);
        for (int i = 0; i < n; i++)
            r.words[i] = exclusive ? (words[i] ^ other.words[i]) : (words[i] | other.words[i]);
        for (int i = n; i < numWords; i++) r.words[i] = words[i];
        for (int i = n; i < other.numWords; i++) r.words[i] = other.words[i];
        return r;
    }
};

#endif  // OLIVE_BITMAP_H
