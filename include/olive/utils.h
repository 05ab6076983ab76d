/*
 * olive_b200 source-compatible header layer: util:: helpers with the
 * reference's names (utils.h:45-172).
 *
 * kernelConfig keeps its signature; it no longer caps the grid at 65,535
 * blocks (the cap dropped vertices past 2^24 in the reference's
 * non-grid-stride kernels, utils.h:68).  The peer-access helpers are kept
 * for source compatibility; the single-GPU engine never calls them.
 */
#ifndef OLIVE_UTILS_H
#define OLIVE_UTILS_H

#include <utility>

#include "common.h"
#include "logging.h"

namespace util {

inline std::pair<int, int> kernelConfig(long long threads,
                                        int threadsPerBlock = DEFAULT_THREADS_PER_BLOCK) {
    if (threads <= 0) return std::make_pair(0, 0);
    assert(threadsPerBlock <= MAX_THREADS_PER_BLOCK);
    if (threads < threadsPerBlock) threadsPerBlock = (int)threads;
    long long blocks = (threads + threadsPerBlock - 1) / threadsPerBlock;
    if (blocks > MAX_BLOCKS) blocks = MAX_BLOCKS;
    return std::make_pair((int)blocks, threadsPerBlock);
}

inline void enablePeerAccess(int self, int other) {
    CUDA_CHECK(cudaSetDevice(self));
    int can = 0;
    CUDA_CHECK(cudaDeviceCanAccessPeer(&can, self, other));
    if (can) {
        CUDA_CHECK(cudaDeviceEnablePeerAccess(other, 0));
        LOG(INFO) << self << " enable peer access " << other;
    } else {
        LOG(WARNING) << self << " cannot access peer " << other;
    }
}

inline void disablePeerAccess(int self, int other) {
    CUDA_CHECK(cudaSetDevice(self));
    int can = 0;
    CUDA_CHECK(cudaDeviceCanAccessPeer(&can, self, other));
    if (can) {
        CUDA_CHECK(cudaDeviceDisablePeerAccess(other));
        LOG(INFO) << self << " disable peer access " << other;
    } else {
        LOG(WARNING) << self << " cannot access peer " << other;
    }
}

inline void enableAllPeerAccess() {
    int n = 0;
    CUDA_CHECK(cudaGetDeviceCount(&n));
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            enablePeerAccess(i, j);
            enablePeerAccess(j, i);
        }
}

inline void disableAllPeerAccess() {
    int n = 0;
    CUDA_CHECK(cudaGetDeviceCount(&n));
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            disablePeerAccess(i, j);
            disablePeerAccess(j, i);
        }
}

inline void expectOverlapOnAllDevices() {
    int n = 0;
    cudaGetDeviceCount(&n);
    for (int i = 0; i < n; i++) {
        int overlap = 0;
        cudaDeviceGetAttribute(&overlap, cudaDevAttrGpuOverlap, i);
        assert(overlap);
    }
}

inline bool isNumeric(const char *str) {
    assert(str);
    for (; *str; str++)
        if (!isdigit((unsigned char)*str)) return false;
    return true;
}

/** xorshift hash of an id (utils.h:165-170), used by the random edge-cut. */
inline size_t hashCode(size_t a) {
    a ^= (a << 13);
    a ^= (a >> 17);
    a ^= (a << 5);
    return a;
}

}  // namespace util

#endif  // OLIVE_UTILS_H
