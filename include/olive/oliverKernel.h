/*
 * olive_b200 source-compatible header layer: the engine kernels behind
 * Oliver<V,E,A>, templated on the application's functors and compiled for
 * sm_100a in the application's translation unit.
 *
 * They replace the reference's five kernels (oliverKernel.h:45-221):
 *   edgeFilter / edgeMap (oliverKernel.h:45-83, 148-178) run on the engine's
 *     shared templates (include/olive_b200/olv_advance.cuh), the same ones the
 *     C ABI's BFS and SSSP instantiate:
 *       push  olv::k_advance_chunks / k_advance_pieces with PushOp: a CTA scans
 *             256 sources' out-degrees and all threads walk the chunk's edges
 *             (rows over kHub edges go to warp pieces); each destination's
 *             bit is set once (a plain load first, the atomic only when it is
 *             clear) and the newly flagged vertex is listed, so the next
 *             vertexFilter reads only the touched vertices;
 *       pull  olv::k_pull_chunks / k_pull_pieces with PullOp over the reverse
 *             graph: each row reduces its in-edges from source-subset members
 *             into a shared-memory slot (the functor's own reduce), then one
 *             store; chosen on the device when the frontier's out-edges pass
 *             E / pull_div (default 1; or always / never, OLIVE_DIRECTION).  A functor
 *             may opt into a narrower pull: `pullCandidate(const V &)` skips
 *             rows, `static constexpr bool pullFirstHit` stops a row at its
 *             first contribution (valid when any one contribution is enough,
 *             as for BFS levels): the pull then runs k_pull_first_rows /
 *             k_pull_first_long (a thread per row probes the row's likeliest
 *             parent, the in-neighbour of most out-edges found once by
 *             readGraph; rows it fails go to 8-lane groups that scan their
 *             in-edges; early exit) and is chosen from E / (pull_div * 16)
 *             frontier out-edges.
 *   k_vertex_filter  flags -> queue with cond/update (oliverKernel.h:85-141):
 *     over the listed members (or the bitmap when no list is known); ballot
 *     compaction into a shared-memory stage, one queue atomic per flush;
 *     writes the queue, its bitmap and the sum of the kept vertices'
 *     out-degrees.  cond receives the vertex's
 *     accumulator -- the reference passed the vertex id (oliverKernel.h:112,
 *     135), which SSSP.cu's cond cannot use.
 *   k_vertex_map  (oliverKernel.h:184-221), over queue, list or bitmap.
 * Every kernel is grid-stride (the reference's 65,535-block cap skipped
 * vertices past 2^24, utils.h:68).  Empty edge types (Dump_Edge) take no
 * storage: the functor receives a local default-constructed value.
 */
#ifndef OLIVE_OLIVER_KERNEL_H
#define OLIVE_OLIVER_KERNEL_H

#include <type_traits>

#include "../olive_b200/olv_advance.cuh"
#include "common.h"
#include "vertexSubset.h"

namespace olive_detail {

constexpr int kT = 256;            // threads per CTA (olv::kBlock)
constexpr uint32_t kHub = 1024;    // push: rows with more out-edges go to pieces
constexpr uint32_t kPiece = 1024;
constexpr uint32_t kPullHub = 4096;   // pull: rows with more in-edges go to pieces
constexpr uint32_t kPullPiece = 2048;
constexpr double kFirstHitPullFactor = 16.0;  // pull at E / (pull_div * 16) for first-hit ops
constexpr uint32_t kModePush = 0;
constexpr uint32_t kModePull = 1;

__device__ __forceinline__ uint32_t lane() { return threadIdx.x & 31; }

template <typename E>
__device__ __forceinline__ E &edge_ref(E *vals, EdgeId e, E &dummy) {
    if constexpr (std::is_empty<E>::value) {
        return dummy;
    } else {
        return vals[e];
    }
}

__device__ __forceinline__ bool bit_of(const Word *bits, VertexId v) {
    return (bits[v >> 6] >> (v & 63)) & 1;
}

// Set v's bit; true when this call set it.  A plain load first: most
// destinations reached again in a superstep are already flagged.
__device__ __forceinline__ bool set_bit(Word *bits, VertexId v) {
    const Word m = (Word)1 << (v & 63);
    if (__ldcg(&bits[v >> 6]) & m) return false;
    const unsigned long long old =
        atomicOr(reinterpret_cast<unsigned long long *>(&bits[v >> 6]), (unsigned long long)m);
    return !(old & m);
}

// ------------------------------------------------- functor opt-in traits --
template <class F, class V, class = void>
struct has_pull_candidate : std::false_type {};
template <class F, class V>
struct has_pull_candidate<
    F, V, std::void_t<decltype(std::declval<F &>().pullCandidate(std::declval<const V &>()))>>
    : std::true_type {};

template <class F, class = void>
struct pull_first_hit : std::false_type {};
template <class F>
struct pull_first_hit<F, std::void_t<decltype(F::pullFirstHit)>>
    : std::integral_constant<bool, F::pullFirstHit> {};

// ------------------------------------------------------------------ push --
// Op for olv::k_advance_chunks / k_advance_pieces: gather + reduce per edge,
// flag and list each destination once.
template <class V, class A, class E, class F, bool MarkDst>
struct PushOp {
    static constexpr int kMinBlocks = 2;
    static constexpr bool kHasFar = false;
    static constexpr bool kPacked = false;
    using SV = uint32_t;   // the source id: gather reads its value and degree
    struct Pre {
        A x;
    };
    F f;
    const VertexId *outdeg;
    V *vvals;
    A *acc;
    E *evals;
    Word *dbits;   // destination flags (MarkDst) or the engine's written-accumulator flags
    __device__ __forceinline__ void begin(olv::TravCtl *) {}
    __device__ __forceinline__ SV src_value(uint32_t u) const { return u; }
    __device__ __forceinline__ bool on_input(uint32_t) const { return true; }
    __device__ __forceinline__ Pre prepare(uint32_t u, uint32_t e, uint32_t) {
        E dummy{};
        E &ev = edge_ref(evals, e, dummy);
        return Pre{f.gather(vvals[u], outdeg[u], ev)};
    }
    template <int N>
    __device__ __forceinline__ void apply_n(const Pre (&p)[N], const uint32_t (&v)[N],
                                            int (&act)[N]) {
#pragma unroll
        for (int j = 0; j < N; j++)
            if (act[j]) f.reduce(acc[v[j]], p[j].x);
#pragma unroll
        for (int j = 0; j < N; j++) act[j] = act[j] && set_bit(dbits, v[j]) ? 1 : 0;
    }
    __device__ __forceinline__ void on_push(bool, uint32_t) {}
    __device__ __forceinline__ void flush(unsigned long long) {}
};

// ------------------------------------------------------------------ pull --
template <class V, class A, class E, class F>
struct PullOp {
    static constexpr int kMinBlocks = 2;
    static constexpr bool kFirstHit = pull_first_hit<F>::value;
    using Acc = A;
    F f;
    const VertexId *outdeg;
    const EdgeId *eid;      // CSR position of each in-edge (edge values)
    const Word *sbits;      // source subset
    V *vvals;
    A *acc;
    E *evals;
    Word *dbits;
    __device__ __forceinline__ bool row_wanted(uint32_t r) {
        if constexpr (has_pull_candidate<F, V>::value)
            return f.pullCandidate(vvals[r]);
        else
            return true;
    }
    __device__ __forceinline__ A acc_load(uint32_t r) const { return acc[r]; }
    __device__ __forceinline__ bool contributes(uint32_t u, uint32_t e, A &x) {
        if (!bit_of(sbits, u)) return false;
        x = contribution(u, e);
        return true;
    }
    // split form for the first-hit kernels: membership loads first, one gather
    __device__ __forceinline__ bool passes(uint32_t u) const { return bit_of(sbits, u); }
    __device__ __forceinline__ A contribution(uint32_t u, uint32_t e) {
        E dummy{};
        E &ev = edge_ref(evals, eid[e], dummy);
        return f.gather(vvals[u], outdeg[u], ev);
    }
    __device__ __forceinline__ void reduce_slot(A &slot, const A &x) { f.reduce(slot, x); }
    __device__ __forceinline__ void reduce_row(uint32_t r, const A &x) { f.reduce(acc[r], x); }
    __device__ __forceinline__ void store(uint32_t r, const A &slot) { acc[r] = slot; }
    __device__ __forceinline__ bool mark(uint32_t r) { return set_bit(dbits, r); }
    // rows r0..r0+31 (r0 a multiple of 32) with bits in m, flagged with one
    // atomic; the rows whose flags this call set
    __device__ __forceinline__ uint32_t mark_warp(uint32_t r0, uint32_t m) {
        const uint32_t sh = r0 & 63;
        const unsigned long long old = atomicOr(
            reinterpret_cast<unsigned long long *>(&dbits[r0 >> 6]), (unsigned long long)m << sh);
        return m & ~(uint32_t)(old >> sh);
    }
};

// --------------------------------------------------------- edge pass glue --
// Before a pass: the source count and the push/pull choice go into the
// control block (no host round trip).  policy: 0 push, 1 pull, 2 by size.
__global__ void k_edge_setup(olv::TravCtl *c, const SubsetMeta *src, int policy,
                             unsigned long long pull_edges) {
    olv::TravCtl t = {};
    t.qsize[0] = src->qsize;
    const unsigned long long m = src->outEdges;
    bool pull = policy == 1 || (policy == 2 && m != kUnknownEdges && m >= pull_edges);
    t.mode = pull ? kModePull : kModePush;
    *c = t;
}

// After a pass: the destination's list length, its metadata, and the list
// of written accumulators for the next reset.
__global__ void k_edge_finish(const olv::TravCtl *c, SubsetMeta *dst, const VertexId *list,
                              VertexId *accList, SubsetMeta *accMeta) {
    const VertexId n = c->qsize[1];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (dst) {
            dst->qsize = n;
            dst->listValid = 1;
            dst->outEdges = kUnknownEdges;
        }
        accMeta->qsize = n;
        accMeta->listValid = 1;
    }
    if (accList != list)
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
             i += (size_t)gridDim.x * blockDim.x)
            accList[i] = list[i];
}

// Accumulators back to the default: the ones the last pass wrote when they
// are listed, all of them otherwise (the reference refilled all V on the host
// and copied them every superstep, oliver.h:66,127).
template <typename A>
__global__ void k_acc_reset(A *acc, VertexId n, A x, const VertexId *list, SubsetMeta *m) {
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    if (m->listValid) {
        const VertexId k = m->qsize;
        for (size_t i = tid; i < k; i += stride) acc[list[i]] = x;
    } else {
        for (size_t v = tid; v < n; v += stride) acc[v] = x;
    }
}

__global__ void k_meta_set(SubsetMeta *m, VertexId qsize, uint32_t listValid) {
    m->qsize = qsize;
    m->listValid = listValid;
}

// Members of a flag subset without a list, written as a list (the bitmap in
// order), with the sum of their out-degrees.
__global__ void k_bits_to_list(const Word *bits, VertexId n, const VertexId *outdeg,
                               VertexId *list, SubsetMeta *m) {
    unsigned long long deg = 0;
    for (size_t base = blockIdx.x * (size_t)blockDim.x; base < n;
         base += (size_t)gridDim.x * blockDim.x) {
        const size_t v = base + threadIdx.x;
        const bool in = v < n && bit_of(bits, (VertexId)v);
        if (in) deg += outdeg[v];
        olv::warp_push(in, (uint32_t)v, list, &m->qsize);
    }
    olv::warp_add64(deg, &m->outEdges);
}

__global__ void k_meta_zero_for_list(SubsetMeta *m) {
    m->qsize = 0;
    m->outEdges = 0;
}

__global__ void k_meta_list_done(SubsetMeta *m) { m->listValid = 1; }

// vertexFilter: members of src with cond(value, acc) are updated and queued.
template <typename V, typename A, typename F>
__global__ void __launch_bounds__(kT)
k_vertex_filter(const Word *sbits, const VertexId *slist, const SubsetMeta *smeta, VertexId n,
                const VertexId *outdeg, V *vvals, A *acc, VertexId *queue, Word *qbits,
                SubsetMeta *qmeta, F f) {
    const bool listed = smeta->listValid;
    const size_t count = listed ? smeta->qsize : n;
    // the queue staged in shared memory: one counter atomic per flush
    __shared__ uint32_t s_q[olv::kStage];
    __shared__ uint32_t s_qn, s_qlim, s_base;
    __shared__ unsigned long long s_deg;
    if (threadIdx.x == 0) {
        s_qn = 0;
        s_qlim = olv::kStage;
        s_deg = 0;
    }
    __syncthreads();
    unsigned long long deg = 0;
    for (size_t base = blockIdx.x * (size_t)kT; base < count; base += (size_t)gridDim.x * kT) {
        const size_t i = base + threadIdx.x;
        bool keep = false;
        VertexId v = 0;
        if (i < count) {
            v = listed ? slist[i] : (VertexId)i;
            if (listed || bit_of(sbits, v)) {
                A a = acc[v];
                if (f.cond(vvals[v], a)) {
                    f.update(vvals[v], a);
                    keep = true;
                    deg += outdeg[v];
                }
            }
        }
        if (keep)
            atomicOr(reinterpret_cast<unsigned long long *>(&qbits[v >> 6]),
                     (unsigned long long)((Word)1 << (v & 63)));
        const uint32_t vv[1] = {v};
        const int ak[1] = {keep ? 1 : 0};
        olv::stage_push_n<1>(ak, vv, 1, s_q, &s_qn, &s_qlim, olv::kStage, queue, &qmeta->qsize);
        __syncthreads();
        if (min(s_qn, s_qlim) >= olv::kStage / 2)
            olv::stage_flush(s_q, &s_qn, &s_qlim, &s_base, queue, &qmeta->qsize);
        __syncthreads();
    }
    olv::stage_flush(s_q, &s_qn, &s_qlim, &s_base, queue, &qmeta->qsize);
    // the out-degree sum: one global atomic per CTA
    olv::warp_add64(deg, &s_deg);
    __syncthreads();
    if (threadIdx.x == 0 && s_deg) atomicAdd(&qmeta->outEdges, s_deg);
}

// vertexMap over a queue, a listed flag subset or the bitmap.
template <typename V, typename A, typename F>
__global__ void k_vertex_map(const Word *bits, const VertexId *list, const SubsetMeta *m,
                             bool dense, VertexId n, V *vvals, A *acc, F f) {
    const bool listed = dense || m->listValid;
    const size_t count = listed ? m->qsize : n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x) {
        const VertexId v = listed ? list[i] : (VertexId)i;
        if (listed || bit_of(bits, v)) f(vvals[v], acc[v]);
    }
}

// ------------------------------------------------------ graph preparation --
__global__ void k_out_degrees(const EdgeId *rowptr, VertexId n, VertexId *outdeg) {
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < n;
         v += (size_t)gridDim.x * blockDim.x)
        outdeg[v] = rowptr[v + 1] - rowptr[v];
}

__global__ void k_row_of_edge(const EdgeId *rowptr, VertexId n, VertexId *src) {
    const size_t w = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t v = w; v < n; v += nw)
        for (EdgeId e = rowptr[v] + lane(); e < rowptr[v + 1]; e += 32) src[e] = (VertexId)v;
}

__global__ void k_iota(EdgeId *a, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        a[i] = (EdgeId)i;
}

__global__ void k_in_degrees(const VertexId *col, size_t E, VertexId *indeg) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < E;
         i += (size_t)gridDim.x * blockDim.x)
        atomicAdd(&indeg[col[i]], 1u);
}

// Each vertex's likeliest parent for first-hit pulls: the in-edge whose
// source has the most out-edges (the earliest CSC position among equals),
// kept as the maximum of (out-degree << 32 | ~position).  dst holds the
// destination of each CSC position (sorted), so a warp's lanes with one
// destination are adjacent: a segmented maximum in the warp, then one
// atomicMax per destination run.
__global__ void k_first_parent_max(const VertexId *dst, const VertexId *src, const VertexId *outdeg,
                                   size_t E, unsigned long long *best) {
    const uint32_t ln = lane();
    for (size_t base = blockIdx.x * (size_t)blockDim.x; base < E;
         base += (size_t)gridDim.x * blockDim.x) {
        const size_t i = base + threadIdx.x;
        const bool valid = i < E;
        const VertexId v = valid ? dst[i] : 0xffffffffu;
        unsigned long long key =
            valid ? (unsigned long long)outdeg[src[i]] << 32 | (uint32_t)~(uint32_t)i : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long k2 = __shfl_down_sync(0xffffffffu, key, o);
            const VertexId v2 = __shfl_down_sync(0xffffffffu, v, o);
            if (ln + o < 32 && v2 == v && k2 > key) key = k2;
        }
        const VertexId vp = __shfl_up_sync(0xffffffffu, v, 1);
        if (valid && (ln == 0 || vp != v) && __ldcg(&best[v]) < key) atomicMax(&best[v], key);
    }
}

__global__ void k_first_parent_set(const unsigned long long *best, const VertexId *src, size_t n,
                                   VertexId *first, EdgeId *firstpos) {
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < n;
         v += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long b = best[v];
        const EdgeId pos = (EdgeId)~(uint32_t)b;
        first[v] = (b >> 32) ? src[pos] : olv::kNoFirst;
        firstpos[v] = (b >> 32) ? pos : 0;
    }
}

__global__ void k_gather_u32(const VertexId *in, const EdgeId *idx, size_t n, VertexId *out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = in[idx[i]];
}

}  // namespace olive_detail

#endif  // OLIVE_OLIVER_KERNEL_H
