/*
 * olive_b200 source-compatible header layer: VertexSubset
 * (vertexSubset.h:38-156).  As in the reference, isDense == true means the
 * subset is a queue of ids and isDense == false means a per-vertex flag
 * array (the names are inverted relative to the usual meaning;
 * vertexSubset.h:41-44).  Flags are one byte per vertex on the device;
 * the queue length lives on the device, with a pinned host copy that
 * size() refreshes.  The caller frees with del(), as in the reference.
 */
#ifndef OLIVE_VERTEX_SUBSET_H
#define OLIVE_VERTEX_SUBSET_H

#include "common.h"

class VertexSubset {
public:
    bool isDense;
    VertexId n;
    uint8_t *flags;          // sparse (flag) representation, device
    VertexId *queue;         // dense (queue) representation, device
    VertexId *qSizeDevice;   // queue length, device
    VertexId *qSize;         // queue length, pinned host copy

    VertexSubset()
        : isDense(false), n(0), flags(NULL), queue(NULL), qSizeDevice(NULL), qSize(NULL) {}

    /** Flag subset of n vertices, universal or empty. */
    VertexSubset(VertexId n_, bool universal)
        : isDense(false), n(n_), flags(NULL), queue(NULL), qSizeDevice(NULL), qSize(NULL) {
        CUDA_CHECK(cudaMalloc((void **)&flags, n_ ? n_ : 1));
        CUDA_CHECK(cudaMemset(flags, universal ? 1 : 0, n_));
    }

    /** Empty queue subset with room for n vertices. */
    explicit VertexSubset(VertexId n_)
        : isDense(true), n(n_), flags(NULL), queue(NULL), qSizeDevice(NULL), qSize(NULL) {
        allocQueue();
        *qSize = 0;
        CUDA_CHECK(cudaMemset(qSizeDevice, 0, sizeof(VertexId)));
    }

    /** Queue subset holding the single vertex v. */
    VertexSubset(VertexId n_, VertexId v)
        : isDense(true), n(n_), flags(NULL), queue(NULL), qSizeDevice(NULL), qSize(NULL) {
        allocQueue();
        CUDA_CHECK(cudaMemcpy(queue, &v, sizeof(VertexId), cudaMemcpyHostToDevice));
        *qSize = 1;
        CUDA_CHECK(cudaMemcpy(qSizeDevice, qSize, sizeof(VertexId), cudaMemcpyHostToDevice));
    }

    /** Queue length (blocking read of the device counter). */
    inline VertexId size() const {
        assert(isDense);
        CUDA_CHECK(cudaMemcpy(qSize, qSizeDevice, sizeof(VertexId), cudaMemcpyDeviceToHost));
        return *qSize;
    }

    inline VertexId capacity() const { return n; }

    inline void clear() {
        if (isDense) {
            *qSize = 0;
            CUDA_CHECK(cudaMemsetAsync(qSizeDevice, 0, sizeof(VertexId)));
        } else {
            CUDA_CHECK(cudaMemsetAsync(flags, 0, n));
        }
    }

    inline void print() {
        if (isDense) {
            VertexId k = size();
            VertexId *h = new VertexId[k ? k : 1];
            CUDA_CHECK(cudaMemcpy(h, queue, k * sizeof(VertexId), cudaMemcpyDeviceToHost));
            printf("dense: ");
            for (VertexId i = 0; i < k; i++) printf("%u ", h[i]);
            printf("\n");
            delete[] h;
        } else {
            uint8_t *h = new uint8_t[n ? n : 1];
            CUDA_CHECK(cudaMemcpy(h, flags, n, cudaMemcpyDeviceToHost));
            printf("sparse: ");
            for (VertexId i = 0; i < n; i++)
                if (h[i]) printf("%u ", i);
            printf("\n");
            delete[] h;
        }
    }

    void del() {
        if (flags) cudaFree(flags);
        if (queue) cudaFree(queue);
        if (qSizeDevice) cudaFree(qSizeDevice);
        if (qSize) cudaFreeHost(qSize);
        flags = NULL;
        queue = NULL;
        qSizeDevice = NULL;
        qSize = NULL;
    }

private:
    void allocQueue() {
        CUDA_CHECK(cudaMalloc((void **)&queue, (size_t)(n ? n : 1) * sizeof(VertexId)));
        CUDA_CHECK(cudaMalloc((void **)&qSizeDevice, sizeof(VertexId)));
        CUDA_CHECK(cudaMallocHost((void **)&qSize, sizeof(VertexId)));
    }
};

#endif  // OLIVE_VERTEX_SUBSET_H
