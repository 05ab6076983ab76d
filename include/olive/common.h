/*
 * olive_b200 source-compatible header layer: common types and macros.
 *
 * Same names and meaning as the reference's common.h (common.h:55-130):
 * VertexId/EdgeId/PartitionId are uint32, Dump_Edge is the empty edge type,
 * THREAD_INDEX/NUM_THREADS, CUDA_CHECK, H2D/D2H, Managed.
 *
 * Differences, on purpose:
 *   - no atomicAdd(double*, double) is defined: CUDA provides it natively on
 *     sm_60 and later, and the reference's CAS version (common.h:141-150)
 *     clashes with it (the reference does not build with CUDA 12.9);
 *   - MAX_BLOCKS is the sm_100a grid limit; every kernel of this layer is
 *     grid-stride, so no vertex is dropped at V > 2^24 (the reference's
 *     65,535-block cap with non-grid-stride kernels skipped the tail,
 *     utils.h:68 with oliverKernel.h:100,164,196).
 */
#ifndef OLIVE_COMMON_H
#define OLIVE_COMMON_H

#include <assert.h>
#include <ctype.h>
#include <inttypes.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cuda_runtime.h"

typedef uint64_t Word;
typedef uint32_t VertexId;
typedef uint32_t EdgeId;
typedef uint32_t PartitionId;

struct Dump_Edge {};

const int DEFAULT_THREADS_PER_BLOCK = 256;
const int MAX_THREADS_PER_BLOCK = 1024;
const int MAX_BLOCKS = 2147483647;

#define BLOCK_INDEX blockIdx.x
#define THREAD_INDEX (threadIdx.x + blockDim.x * blockIdx.x)
#define NUM_BLOCKS gridDim.x
#define NUM_THREADS (blockDim.x * gridDim.x)

#define CUDA_CHECK(cuda_call)                                                        \
    do {                                                                             \
        cudaError_t err_ = (cuda_call);                                              \
        if (err_ != cudaSuccess) {                                                   \
            fprintf(stderr, "CUDA Error in file '%s' in line %i : %s.\n", __FILE__,  \
                    __LINE__, cudaGetErrorString(err_));                             \
            assert(false);                                                           \
            abort();                                                                 \
        }                                                                            \
    } while (0);

#define H2D(dst, src, size) cudaMemcpy(dst, src, size, cudaMemcpyHostToDevice)
#define D2H(dst, src, size) cudaMemcpy(dst, src, size, cudaMemcpyDeviceToHost)

class Managed {
public:
    void *operator new(size_t len) {
        void *ptr;
        CUDA_CHECK(cudaMallocManaged(&ptr, len));
        return ptr;
    }
    void operator delete(void *ptr) { CUDA_CHECK(cudaFree(ptr)); }
};

#endif  // OLIVE_COMMON_H
