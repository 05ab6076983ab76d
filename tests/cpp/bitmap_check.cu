// Exercises the source-compatible Bitmap (include/olive/bitmap.h) on the GPU:
// concurrent atomic set/unset from device threads, host get/count, the
// reference's &, |, ^ operators and copy semantics.  Prints "bitmap ok" and
// exits 0 when every check holds.  Built and run by tests/test_gpu_bitmap.py.
#include <cstdio>
#include <cstdlib>

#include "bitmap.h"

#define EXPECT(c)                                                    \
    do {                                                             \
        if (!(c)) {                                                  \
            fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c); \
            return 1;                                                \
        }                                                            \
    } while (0)

__global__ void k_set(Bitmap *b, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (i % 3 == 0) b->set(i);
}

__global__ void k_unset(Bitmap *b, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (i % 9 == 0) b->unset(i);
}

__global__ void k_count(const Bitmap *b, int n, unsigned long long *c) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (b->get(i)) atomicAdd(c, 1ull);
}

int main() {
    const int n = 100003;
    Bitmap *b = new Bitmap(n);   // Managed: the object itself is reachable from kernels
    EXPECT(b->capacity() == ((n - 1) / 64 + 1) * 64);
    k_set<<<64, 256>>>(b, n);
    k_unset<<<64, 256>>>(b, n);
    CUDA_CHECK(cudaDeviceSynchronize());
    size_t want = 0;
    for (int i = 0; i < n; i++) {
        const bool w = i % 3 == 0 && i % 9 != 0;
        want += w;
        EXPECT(b->get(i) == w);
    }
    EXPECT(b->count() == want);
    unsigned long long *c;
    CUDA_CHECK(cudaMallocManaged(&c, sizeof *c));
    *c = 0;
    k_count<<<64, 256>>>(b, n, c);
    CUDA_CHECK(cudaDeviceSynchronize());
    EXPECT(*c == want);
    cudaFree(c);
    delete b;

    Bitmap x(200), y(64);    // 4 words and 1 word
    x.set(5);
    x.set(150);
    y.set(5);
    y.set(7);
    Bitmap a = x & y, o = x | y, e = x ^ y;
    EXPECT(a.capacity() == 256 && o.capacity() == 256 && e.capacity() == 256);
    EXPECT(a.get(5) && !a.get(7) && !a.get(150) && a.count() == 1);
    EXPECT(o.get(5) && o.get(7) && o.get(150) && o.count() == 3);
    EXPECT(!e.get(5) && e.get(7) && e.get(150) && e.count() == 2);
    Bitmap h;
    h = x;                    // deep copy
    h.unset(5);
    EXPECT(x.get(5) && !h.get(5) && h.get(150));
    Bitmap m(std::move(h));
    EXPECT(m.get(150) && h.capacity() == 0);
    x.clear();
    EXPECT(x.count() == 0 && x.capacity() == 256);
    printf("bitmap ok\n");
    return 0;
}
