/*
 * olive_b200 source-compatible header layer: VertexSubset
 * (vertexSubset.h:38-156).  As in the reference, isDense == true means the
 * subset is a queue of ids and isDense == false means the flag
 * representation (the names are inverted relative to the usual meaning;
 * vertexSubset.h:41-44).
 *
 * Both representations carry a bitmap of the members in 64-bit words
 * (`bits`, V/8 bytes: 2 MB at 2^24 vertices, L2-resident) next to a list of
 * the members (`queue`):
 *   - queue subsets: `queue[0, size)` holds the members, and their bits are
 *     set, so an edgeFilter can test source membership for a pull;
 *   - flag subsets: the bitmap is authoritative; `queue` lists the members
 *     when the list is known (an edgeFilter's output lists every vertex it
 *     flags), so vertexFilter, vertexMap and clear() touch only those, and
 *     fall back to a pass over the bitmap otherwise (the universal subset).
 * The reference kept one int flag per vertex (4 B) and scanned all V of them
 * in every vertexFilter.  Alongside the size, the device metadata keeps the
 * sum of the members' out-degrees when vertexFilter built the queue, which
 * the next edgeFilter uses to choose push or pull.  The caller frees with
 * del(), as in the reference.
 */
#ifndef OLIVE_VERTEX_SUBSET_H
#define OLIVE_VERTEX_SUBSET_H

#include "common.h"

namespace olive_detail {

// Device-side description of a subset, read and written by the engine kernels.
struct SubsetMeta {
    VertexId qsize;               // entries in the member list
    uint32_t listValid;           // flag subsets: the list holds every member
    unsigned long long outEdges;  // sum of the members' out-degrees (~0: unknown)
};

constexpr unsigned long long kUnknownEdges = ~0ull;

__global__ void k_subset_set_one(Word *bits, VertexId *queue, SubsetMeta *m, VertexId v) {
    bits[v >> 6] |= (Word)1 << (v & 63);
    queue[0] = v;
    m->qsize = 1;
    m->listValid = 1;
    m->outEdges = kUnknownEdges;
}

// Clear the members: only the words of listed members when the list is known
// and short, every word otherwise.  One launch; every thread reads the same
// metadata, so the choice is uniform.
__global__ void k_subset_clear(Word *bits, size_t words, const VertexId *queue, SubsetMeta *m) {
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const VertexId n = m->qsize;
    if (m->listValid && (size_t)n * 4 < words) {
        for (size_t i = tid; i < n; i += stride) bits[queue[i] >> 6] = 0;
    } else {
        for (size_t w = tid; w < words; w += stride) bits[w] = 0;
    }
}

__global__ void k_subset_reset_meta(SubsetMeta *m) {
    m->qsize = 0;
    m->listValid = 1;
    m->outEdges = 0;
}

}  // namespace olive_detail

class VertexSubset {
public:
    bool isDense;                       // true: queue of ids; false: flags
    VertexId n;
    Word *bits;                         // members as a bitmap, device
    VertexId *queue;                    // members as a list, device
    VertexId *qSizeDevice;              // list length, device (inside meta)
    VertexId *qSize;                    // list length, pinned host copy
    olive_detail::SubsetMeta *meta;     // device metadata
    olive_detail::SubsetMeta *hostMeta; // pinned host copy (size() refreshes it)
    bool listKnown;                     // host view: the device list holds every member

    VertexSubset()
        : isDense(false), n(0), bits(NULL), queue(NULL), qSizeDevice(NULL), qSize(NULL),
          meta(NULL), hostMeta(NULL), listKnown(true) {}

    /** Flag subset of n vertices, universal or empty. */
    VertexSubset(VertexId n_, bool universal) : isDense(false), n(n_) {
        alloc();
        if (universal) {
            // every bit of the first n set, the rest of the last word clear
            CUDA_CHECK(cudaMemset(bits, 0xff, words() * sizeof(Word)));
            if (n_ & 63) {
                const Word last = ((Word)1 << (n_ & 63)) - 1;
                CUDA_CHECK(cudaMemcpy(bits + words() - 1, &last, sizeof last,
                                      cudaMemcpyHostToDevice));
            }
            olive_detail::SubsetMeta h = {0, 0, olive_detail::kUnknownEdges};
            CUDA_CHECK(cudaMemcpy(meta, &h, sizeof h, cudaMemcpyHostToDevice));
            listKnown = false;
        }
    }

    /** Empty queue subset with room for n vertices. */
    explicit VertexSubset(VertexId n_) : isDense(true), n(n_) { alloc(); }

    /** Queue subset holding the single vertex v. */
    VertexSubset(VertexId n_, VertexId v) : isDense(true), n(n_) {
        alloc();
        olive_detail::k_subset_set_one<<<1, 1>>>(bits, queue, meta, v);
        CUDA_CHECK(cudaGetLastError());
        *qSize = 1;
    }

    /** Queue length (blocking read of the device counter). */
    inline VertexId size() const {
        assert(isDense);
        CUDA_CHECK(cudaMemcpy(hostMeta, meta, sizeof *meta, cudaMemcpyDeviceToHost));
        return *qSize;
    }

    inline VertexId capacity() const { return n; }

    inline size_t words() const { return ((size_t)n + 63) / 64; }

    /** Remove every member (device-side, stream ordered). */
    inline void clear() {
        if (!n) return;
        olive_detail::k_subset_clear<<<gridFor(words()), 256>>>(bits, words(), queue, meta);
        olive_detail::k_subset_reset_meta<<<1, 1>>>(meta);
        CUDA_CHECK(cudaGetLastError());
        *qSize = 0;
        listKnown = true;
    }

    /** Member test on the host (copies one word). */
    inline bool contains(VertexId v) const {
        Word w = 0;
        CUDA_CHECK(cudaMemcpy(&w, bits + (v >> 6), sizeof w, cudaMemcpyDeviceToHost));
        return (w >> (v & 63)) & 1;
    }

    inline void print() {
        Word *h = new Word[words() ? words() : 1];
        CUDA_CHECK(cudaMemcpy(h, bits, words() * sizeof(Word), cudaMemcpyDeviceToHost));
        printf(isDense ? "dense: " : "sparse: ");
        if (isDense) {
            VertexId k = size();
            VertexId *q = new VertexId[k ? k : 1];
            CUDA_CHECK(cudaMemcpy(q, queue, k * sizeof(VertexId), cudaMemcpyDeviceToHost));
            for (VertexId i = 0; i < k; i++) printf("%u ", q[i]);
            delete[] q;
        } else {
            for (VertexId i = 0; i < n; i++)
                if ((h[i >> 6] >> (i & 63)) & 1) printf("%u ", i);
        }
        printf("\n");
        delete[] h;
    }

    void del() {
        if (bits) cudaFree(bits);
        if (queue) cudaFree(queue);
        if (meta) cudaFree(meta);
        if (hostMeta) cudaFreeHost(hostMeta);
        bits = NULL;
        queue = NULL;
        meta = NULL;
        hostMeta = NULL;
        qSizeDevice = NULL;
        qSize = NULL;
    }

    static unsigned gridFor(size_t items) {
        size_t b = (items + 255) / 256;
        return (unsigned)(b < 1 ? 1 : (b > 2368 ? 2368 : b));
    }

private:
    void alloc() {
        CUDA_CHECK(cudaMalloc((void **)&bits, (words() ? words() : 1) * sizeof(Word)));
        CUDA_CHECK(cudaMemset(bits, 0, (words() ? words() : 1) * sizeof(Word)));
        CUDA_CHECK(cudaMalloc((void **)&queue, (size_t)(n ? n : 1) * sizeof(VertexId)));
        CUDA_CHECK(cudaMalloc((void **)&meta, sizeof(olive_detail::SubsetMeta)));
        CUDA_CHECK(cudaMemset(meta, 0, sizeof(olive_detail::SubsetMeta)));
        olive_detail::SubsetMeta h = {0, 1, 0};
        CUDA_CHECK(cudaMemcpy(meta, &h, sizeof h, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMallocHost((void **)&hostMeta, sizeof(olive_detail::SubsetMeta)));
        *hostMeta = h;
        qSizeDevice = &meta->qsize;
        qSize = &hostMeta->qsize;
        listKnown = true;
    }
};

#endif  // OLIVE_VERTEX_SUBSET_H
