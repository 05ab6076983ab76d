/*
 * olive_b200 source-compatible header layer: the engine kernels behind
 * Oliver<V,E,A>, templated on the application's functors and compiled for
 * sm_100a in the application's translation unit.
 *
 * They replace the reference's five kernels (oliverKernel.h:45-221):
 *   k_expand / k_expand_pieces   edgeFilter + edgeMap (oliverKernel.h:45-83,
 *        148-178).  Load-balanced: a CTA takes 256 sources (queue entries or
 *        flagged vertices), scans their out-degrees in shared memory and all
 *        256 threads walk the chunk's edges, so column reads are contiguous
 *        runs; rows longer than kHub edges are cut into kPiece-edge pieces that
 *        a second kernel spreads over every warp.  The reference gave each
 *        source a fixed group of 1..32 threads (hubs serialised).
 *   k_vertex_filter   flags -> queue with cond/update (oliverKernel.h:85-141);
 *        grid-stride, one atomic per warp (ballot/popc compaction).  cond
 *        receives the vertex's accumulator -- the reference passed the vertex
 *        id (oliverKernel.h:112,135), which SSSP.cu's cond cannot use.
 *   k_vertex_map_dense / k_vertex_map_sparse   (oliverKernel.h:184-221),
 *        grid-stride.
 * Empty edge types (Dump_Edge) take no storage: the functor receives a local
 * default-constructed value.
 */
#ifndef OLIVE_OLIVER_KERNEL_H
#define OLIVE_OLIVER_KERNEL_H

#include <type_traits>

#include "common.h"

namespace olive_detail {

constexpr int kT = 256;          // threads per CTA
constexpr uint32_t kHub = 4096;  // rows longer than this are split into pieces
constexpr uint32_t kPiece = 2048;

__device__ __forceinline__ uint32_t lane() { return threadIdx.x & 31; }

template <typename E>
__device__ __forceinline__ E &edge_ref(E *vals, EdgeId e, E &dummy) {
    if constexpr (std::is_empty<E>::value) {
        return dummy;
    } else {
        return vals[e];
    }
}

__device__ __forceinline__ void warp_append(bool p, VertexId v, VertexId *q, VertexId *qsize) {
    const unsigned m = __ballot_sync(0xffffffffu, p);
    if (!m) return;
    const uint32_t leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane() == leader) base = atomicAdd(qsize, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (p) q[base + __popc(m & ((1u << lane()) - 1u))] = v;
}

__device__ __forceinline__ uint32_t cta_exclusive_scan(uint32_t x, uint32_t *total,
                                                       uint32_t *s_warp) {
    const uint32_t ln = lane(), wid = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (ln >= (uint32_t)o) incl += t;
    }
    if (ln == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        constexpr int NW = kT / 32;
        uint32_t t = ln < NW ? s_warp[ln] : 0, ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, ti, o);
            if (ln >= (uint32_t)o) ti += y;
        }
        if (ln < NW) s_warp[ln] = ti - t;
        if (ln == NW - 1) s_warp[32] = ti;
    }
    __syncthreads();
    const uint32_t r = s_warp[wid] + incl - x;
    *total = s_warp[32];
    __syncthreads();
    return r;
}

struct ExpandArgs {
    const VertexId *queue;      // FromQueue: sources
    const VertexId *qsize;
    const uint8_t *srcflags;    // !FromQueue: flag per vertex
    VertexId n;                 // vertex count
    const EdgeId *rowptr;
    const VertexId *col;
    uint8_t *dstflags;          // MarkDst: flags of the destinations
    uint2 *pieces;
    uint32_t *npieces;
};

template <typename V, typename A, typename E, typename F, bool MarkDst>
__device__ __forceinline__ void visit_edge(const ExpandArgs &a, F &f, const V &sv, EdgeId outdeg,
                                           EdgeId e, V *vvals, A *acc, E *evals) {
    E dummy{};
    E &ev = edge_ref(evals, e, dummy);
    const VertexId v = a.col[e];
    A x = f.gather(sv, outdeg, ev);
    f.reduce(acc[v], x);
    if (MarkDst) a.dstflags[v] = 1;
}

template <typename V, typename A, typename E, typename F, bool FromQueue, bool MarkDst>
__global__ void __launch_bounds__(kT)
k_expand(ExpandArgs a, V *vvals, A *acc, E *evals, F f) {
    __shared__ uint32_t s_beg[kT], s_off[kT], s_src[kT];
    __shared__ uint32_t s_warp[33];
    const uint64_t n = FromQueue ? *a.qsize : a.n;
    for (uint64_t chunk = blockIdx.x; chunk * kT < n; chunk += gridDim.x) {
        const uint64_t i = chunk * kT + threadIdx.x;
        uint32_t beg = 0, deg = 0, u = 0;
        if (i < n) {
            u = FromQueue ? a.queue[i] : (VertexId)i;
            if (FromQueue || a.srcflags[u]) {
                beg = a.rowptr[u];
                deg = a.rowptr[u + 1] - beg;
                if (deg > kHub) {
                    const uint32_t np = (deg + kPiece - 1) / kPiece;
                    const uint32_t b = atomicAdd(a.npieces, np);
                    for (uint32_t p = 0; p < np; p++) a.pieces[b + p] = make_uint2(u, p);
                    deg = 0;
                }
            }
        }
        uint32_t total;
        const uint32_t off = cta_exclusive_scan(deg, &total, s_warp);
        s_beg[threadIdx.x] = beg;
        s_off[threadIdx.x] = off;
        s_src[threadIdx.x] = u;
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < total; k += kT) {
            uint32_t lo = 0;
#pragma unroll
            for (uint32_t step = kT / 2; step > 0; step >>= 1)
                if (s_off[lo + step] <= k) lo += step;
            const VertexId src = s_src[lo];
            const EdgeId e = s_beg[lo] + (k - s_off[lo]);
            const EdgeId outdeg = a.rowptr[src + 1] - a.rowptr[src];
            const V sv = vvals[src];
            visit_edge<V, A, E, F, MarkDst>(a, f, sv, outdeg, e, vvals, acc, evals);
        }
        __syncthreads();
    }
}

template <typename V, typename A, typename E, typename F, bool MarkDst>
__global__ void __launch_bounds__(kT)
k_expand_pieces(ExpandArgs a, V *vvals, A *acc, E *evals, F f) {
    const uint32_t np = *a.npieces;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = warp; p < np; p += nwarps) {
        const uint2 pc = a.pieces[p];
        const VertexId u = pc.x;
        const EdgeId rb = a.rowptr[u], re = a.rowptr[u + 1];
        const EdgeId b = rb + pc.y * kPiece;
        const EdgeId end = min(re, b + kPiece);
        const V sv = vvals[u];
        for (EdgeId e = b + lane(); e < end; e += 32)
            visit_edge<V, A, E, F, MarkDst>(a, f, sv, re - rb, e, vvals, acc, evals);
    }
}

template <typename V, typename A, typename F>
__global__ void __launch_bounds__(kT)
k_vertex_filter(const uint8_t *flags, VertexId n, V *vvals, A *acc, VertexId *queue,
                VertexId *qsize, F f) {
    for (uint64_t base = (uint64_t)blockIdx.x * kT; base < n; base += (uint64_t)gridDim.x * kT) {
        const uint64_t v = base + threadIdx.x;
        bool keep = false;
        if (v < n && flags[v] && f.cond(vvals[v], acc[v])) {
            f.update(vvals[v], acc[v]);
            keep = true;
        }
        warp_append(keep, (VertexId)v, queue, qsize);
    }
}

template <typename V, typename A, typename F>
__global__ void k_vertex_map_dense(const VertexId *queue, const VertexId *qsize, V *vvals, A *acc,
                                   F f) {
    const uint64_t n = *qsize;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const VertexId v = queue[i];
        f(vvals[v], acc[v]);
    }
}

template <typename V, typename A, typename F>
__global__ void k_vertex_map_sparse(const uint8_t *flags, VertexId n, V *vvals, A *acc, F f) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x)
        if (flags[v]) f(vvals[v], acc[v]);
}

}  // namespace olive_detail

#endif  // OLIVE_OLIVER_KERNEL_H
