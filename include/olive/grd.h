/*
 * olive_b200 source-compatible header layer: GRD<T>, a buffer with a host and
 * a device copy and the reference's method names (grd.h:43-170).  allTo()
 * fills on the device instead of looping on the host and copying
 * (grd.h:90-97); set() writes one element on both sides.
 */
#ifndef OLIVE_GRD_H
#define OLIVE_GRD_H

#include <iostream>

#include "common.h"

namespace olive_detail {
template <typename T>
__global__ void k_fill(T *p, size_t n, T x) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = x;
}

template <typename T>
inline void device_fill(T *p, size_t n, T x, cudaStream_t s = 0) {
    if (!n) return;
    size_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_fill<T><<<(unsigned)blocks, 256, 0, s>>>(p, n, x);
    CUDA_CHECK(cudaGetLastError());
}
}  // namespace olive_detail

template <typename T>
class GRD {
public:
    T *elemsHost;
    T *elemsDevice;
    size_t length;
    int deviceId;

    GRD() : elemsHost(NULL), elemsDevice(NULL), length(0), deviceId(-1) {}

    __host__ __device__ inline T &operator[](size_t i) const {
#ifdef __CUDA_ARCH__
        return elemsDevice[i];
#else
        return elemsHost[i];
#endif
    }

    inline size_t capacity() const { return length; }

    inline void reserve(size_t len, int id = 0) {
        assert(len > 0 && id >= 0);
        deviceId = id;
        length = len;
        elemsHost = new T[len]();
        CUDA_CHECK(cudaSetDevice(deviceId));
        CUDA_CHECK(cudaMalloc((void **)&elemsDevice, len * sizeof(T)));
    }

    void allTo(T x) {
        for (size_t i = 0; i < length; i++) elemsHost[i] = x;
        CUDA_CHECK(cudaSetDevice(deviceId));
        olive_detail::device_fill(elemsDevice, length, x);
    }

    void clear() { CUDA_CHECK(cudaMemset(elemsDevice, 0, sizeof(T) * length)); }

    void set(size_t i, T x) {
        elemsHost[i] = x;
        CUDA_CHECK(cudaMemcpy(elemsDevice + i, elemsHost + i, sizeof(T), cudaMemcpyDefault));
    }

    inline void persist() {
        if (!length) return;
        CUDA_CHECK(cudaSetDevice(deviceId));
        CUDA_CHECK(cudaMemcpy(elemsHost, elemsDevice, length * sizeof(T), cudaMemcpyDefault));
    }

    inline void print() {
        for (size_t i = 0; i < length; i++) elemsHost[i].print();
    }

    inline void peek() {
        persist();
        for (size_t i = 0; i < length; i++) std::cout << elemsHost[i] << " ";
        printf("\n");
    }

    inline void cache() {
        if (!length) return;
        CUDA_CHECK(cudaSetDevice(deviceId));
        CUDA_CHECK(cudaMemcpy(elemsDevice, elemsHost, length * sizeof(T), cudaMemcpyDefault));
    }

    inline void del() {
        if (deviceId < 0) return;
        delete[] elemsHost;
        if (elemsDevice) {
            CUDA_CHECK(cudaSetDevice(deviceId));
            CUDA_CHECK(cudaFree(elemsDevice));
        }
        elemsHost = NULL;
        elemsDevice = NULL;
        length = 0;
        deviceId = -1;
    }
};

#endif  // OLIVE_GRD_H
