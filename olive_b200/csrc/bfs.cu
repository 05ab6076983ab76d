// Direction-optimising BFS.
//
// Result contract: testBFS.cu:42-87 and BFS.cu:82-160 run to completion --
// int32 level per vertex, 0x7fffffff when unreached, level[src] = 0.
//
// Reference path, per level (BFS.cu:124-148): edgeFilter over the queue
// (oliver.h:56-83: host refill of V accumulators + H2D, edgeFilterKernel with
// a plain-store "benign race", BFS.cu:52-55), then vertexFilter over all V
// flags (oliver.h:92-113) and a blocking D2H of the queue size.
//
// Here each superstep is a fixed chain of kernels that decide on the device
// what to do, so the whole traversal is one CUDA graph launch:
//   k_bfs_begin      choose push or pull from the frontier's edge count
//                    (Beamer's alpha/beta rule), reset the output queue
//   k_advance_chunks push: claim unvisited neighbours with atomicCAS on the
//   k_advance_pieces level array and append them to the next queue (the
//                    claim fuses edgeFilter's reduce and vertexFilter's
//                    cond/update into one step)
//   k_bfs_pull       pull: every unvisited vertex scans its in-edges for a
//                    parent at the current level and stops at the first one
//   k_bfs_end        account edges, swap queues, stop when the queue is empty
#include <stdio.h>

#include <cub/cub.cuh>

#include "olv_advance.cuh"
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"

namespace olv {

struct BfsPushOp {
    using SV = uint32_t;
    static constexpr bool kHasFar = false;
    const uint32_t *rowptr;
    int32_t *level;
    int next;
    unsigned long long acc;
    unsigned long long *m_next;

    __device__ __forceinline__ void begin(TravCtl *c) {
        level = static_cast<int32_t *>(c->vdata);
        next = (int)c->level + 1;
        acc = 0;
        m_next = &c->m_next;
    }
    struct Pre {
        int lvl;
    };
    __device__ __forceinline__ uint32_t src_value(uint32_t) const { return 0; }
    __device__ __forceinline__ Pre prepare(uint32_t, uint32_t, uint32_t v) const {
        return Pre{__ldcg(&level[v])};
    }
    __device__ __forceinline__ int apply(const Pre &p, uint32_t v) {
        if (p.lvl != kInf) return 0;
        return atomicCAS(&level[v], kInf, next) == kInf ? 1 : 0;
    }
    __device__ __forceinline__ void on_push(bool p, uint32_t v) {
        if (p) acc += __ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]);
    }
    __device__ __forceinline__ void flush(unsigned long long) { warp_add64(acc, m_next); }
};

__global__ void k_fill_i32(int32_t *__restrict__ a, uint32_t n, int32_t x) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (reinterpret_cast<uintptr_t>(a) & 15) {   // caller buffer not 16-byte aligned
        for (uint64_t i = tid; i < n; i += stride) a[i] = x;
        return;
    }
    const uint64_t n4 = n / 4;
    int4 *a4 = reinterpret_cast<int4 *>(a);
    for (uint64_t i = tid; i < n4; i += stride) a4[i] = make_int4(x, x, x, x);
    for (uint64_t i = n4 * 4 + tid; i < n; i += stride) a[i] = x;
}

__global__ void k_bfs_init(TravCtl *c, int32_t *level, uint32_t *q0, const uint32_t *rowptr,
                           uint32_t src, unsigned long long E) {
    TravCtl t = {};
    t.qsize[0] = 1;
    t.vdata = level;
    const uint32_t d = rowptr[src + 1] - rowptr[src];
    t.m_f = d;
    t.m_unvisited = E - d;
    *c = t;
    level[src] = 0;
    q0[0] = src;
}

__global__ void k_bfs_begin(TravCtl *c, uint32_t V, float alpha, float beta) {
    if (c->done) return;
    const uint32_t n = c->qsize[c->cur];   // frontier size (queue or bitmap)
    if (n == 0) {
        c->done = 1;
        return;
    }
    if (c->mode == 0) {
        if ((double)c->m_f * alpha > (double)c->m_unvisited) c->mode = 1;
    } else if ((double)n * beta < (double)V) {
        c->mode = 0;
    }
    c->qsize[c->cur ^ 1] = 0;
    c->npieces = 0;
    c->m_next = 0;
    c->reached_pull = 0;
    c->ncand[0] = 0;   // pull overflow list
    if (c->mode == 0 && c->queue_stale) c->qsize[c->cur] = 0;   // rebuilt from the bitmap
}

// Pull-level preparation (pull levels only), two independent index ranges:
//   - bitmap of the current frontier (level == L), one ballot per warp, when the
//     previous level was a push level;
//   - zero the next frontier's bitmap.
struct PullLists {
    uint32_t V;
    const uint32_t *pidx;      // in-edges, highest out-degree source first
    const uint32_t *order;     // vertices by in-degree (heavy: in-degree > kPullHeavy)
    uint32_t n_heavy, n_light;
    uint32_t *cand;            // pull overflow list (V entries)
    uint32_t *fb0, *fb1;
    uint32_t words;            // words per bitmap
};

constexpr uint32_t kPullHeavy = 128;   // in-degree split of the sorted vertex list


__global__ void __launch_bounds__(kBlock)
k_bfs_pull_prep(uint32_t V, TravCtl *c, PullLists p) {
    if (c->done || c->mode != 1) return;
    const int32_t *level = static_cast<const int32_t *>(c->vdata);
    const int L = (int)c->level;
    uint32_t *fcur = c->fb_cur ? p.fb1 : p.fb0;
    uint32_t *fnext = c->fb_cur ? p.fb0 : p.fb1;
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    if (!c->fb_valid)
        for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < V; base += stride) {
            const uint64_t v = base + threadIdx.x;
            const unsigned word = __ballot_sync(0xffffffffu, v < V && __ldcg(&level[v]) == L);
            if (lane_id() == 0) fcur[v >> 5] = word;
        }
    for (uint64_t w = blockIdx.x * (uint64_t)kBlock + threadIdx.x; w < p.words; w += stride)
        fnext[w] = 0;
}

// The current frontier as a queue, from its bitmap, when a push level follows
// a pull level.
__global__ void __launch_bounds__(kBlock)
k_bfs_fb_to_queue(TravCtl *c, uint32_t *q0, uint32_t *q1, PullLists p) {
    if (c->done || c->mode != 0 || !c->queue_stale) return;
    const uint32_t *fb = c->fb_cur ? p.fb1 : p.fb0;
    uint32_t *q = c->cur ? q1 : q0;
    uint32_t *qsz = &c->qsize[c->cur];
    const uint32_t lane = lane_id();
    const uint64_t nw = ((uint64_t)p.V + 31) / 32;
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < nw;
         base += (uint64_t)gridDim.x * kBlock) {
        const uint64_t w = base + threadIdx.x;
        uint32_t bits = w < nw ? fb[w] : 0;
        // one atomic per warp for all the warp's set bits
        const uint32_t cnt = __popc(bits);
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        uint32_t off = 0;
        if (lane == 31 && total) off = atomicAdd(qsz, total);
        off = __shfl_sync(0xffffffffu, off, 31) + incl - cnt;
        while (bits) {
            const uint32_t b = __ffs(bits) - 1;
            bits &= bits - 1;
            q[off++] = (uint32_t)(w * 32 + b);
        }
    }
}

__device__ __forceinline__ bool in_bitmap(const uint32_t *__restrict__ fb, uint32_t u) {
    return (__ldg(&fb[u >> 5]) >> (u & 31)) & 1u;
}

// Pull, pass 1: every unvisited vertex probes its first kProbe1 in-edges (the
// in-edge lists are ordered by source out-degree, so the likeliest parents
// come first) against the frontier bitmap, kParents at a time.  A vertex that
// finds a parent gets level L+1, a bit in the next bitmap and a queue slot;
// one that has more in-edges left goes to the overflow list.  Every thread
// does at most kProbe1 probes, so the lanes of a warp finish together.
constexpr int kParents = 4;
constexpr uint32_t kProbe1 = 8;


__global__ void __launch_bounds__(kBlock)
k_bfs_pull(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowptr,
           TravCtl *c, uint32_t *q0, uint32_t *q1, PullLists p) {
    if (c->done || c->mode != 1) return;
    int32_t *level = static_cast<int32_t *>(c->vdata);
    const int L = (int)c->level;
    const uint32_t *__restrict__ fin = c->fb_cur ? p.fb1 : p.fb0;
    uint32_t *fout = c->fb_cur ? p.fb0 : p.fb1;
    uint32_t *ovf = p.cand;
    const uint32_t lane = lane_id();
    unsigned long long acc = 0, nfound = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < p.V;
         base += (uint64_t)gridDim.x * kBlock) {
        const uint32_t v = (uint32_t)base + threadIdx.x;
        bool found = false, more = false;
        if (v < p.V && level[v] == kInf) {
            const uint32_t b = __ldg(&colptr[v]), e = __ldg(&colptr[v + 1]);
            const uint32_t e1 = e - b > kProbe1 ? b + kProbe1 : e;
            for (uint32_t k = b; k < e1 && !found; k += kParents) {
                uint32_t u[kParents];
#pragma unroll
                for (int j = 0; j < kParents; j++)
                    u[j] = k + j < e1 ? __ldg(&p.pidx[k + j]) : 0xffffffffu;
#pragma unroll
                for (int j = 0; j < kParents; j++)
                    if (u[j] != 0xffffffffu && in_bitmap(fin, u[j])) found = true;
            }
            if (found) {
                level[v] = L + 1;
                acc += __ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]);
            } else {
                more = e1 < e;
            }
        }
        const unsigned word = __ballot_sync(0xffffffffu, found);
        if (lane == 0 && word) atomicOr(&fout[v >> 5], word);
        nfound += found;
        warp_push(more, v, ovf, &c->ncand[0]);
    }
    warp_add64(acc, &c->m_next);
    // the next frontier lives in the bitmap; only its size is counted here
    // (one atomic per warp at the end, not one per iteration)
    warp_add64(nfound, &c->reached_pull);
}

// Pull, pass 2: one warp per overflow vertex scans the rest of its in-edges,
// 32 per probe, and stops at the first parent.
__global__ void __launch_bounds__(kBlock)
k_bfs_pull_overflow(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowptr,
                    TravCtl *c, uint32_t *q0, uint32_t *q1, PullLists p) {
    if (c->done || c->mode != 1) return;
    const uint32_t n = c->ncand[0];
    if (n == 0) return;
    int32_t *level = static_cast<int32_t *>(c->vdata);
    const int L = (int)c->level;
    const uint32_t *__restrict__ fin = c->fb_cur ? p.fb1 : p.fb0;
    uint32_t *fout = c->fb_cur ? p.fb0 : p.fb1;
    const uint32_t lane = lane_id();
    const uint32_t gwarp = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kBlock) >> 5;
    unsigned long long acc = 0, nfound = 0;
    for (uint32_t i = gwarp; i < n; i += nwarps) {
        const uint32_t v = p.cand[i];
        const uint32_t b = __ldg(&colptr[v]) + kProbe1, e = __ldg(&colptr[v + 1]);
        bool found = false;
        for (uint32_t base = b; base < e; base += 32) {
            const uint32_t j = base + lane;
            const bool hit = j < e && in_bitmap(fin, __ldg(&p.pidx[j]));
            if (__any_sync(0xffffffffu, hit)) {
                found = true;
                break;
            }
        }
        if (lane == 0 && found) {
            level[v] = L + 1;
            atomicOr(&fout[v >> 5], 1u << (v & 31));
            acc += __ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]);
            nfound++;
        }
    }
    warp_add64(acc, &c->m_next);
    warp_add64(nfound, &c->reached_pull);
}

__global__ void k_bfs_end(TravCtl *c, cudaGraphConditionalHandle h, int use_cond, uint32_t V) {
    if (!c->done) {
        c->edges_traversed += c->m_f;
        c->reached += c->qsize[c->cur];
        if (c->mode) c->pull_steps++;
        c->m_unvisited -= (c->m_next < c->m_unvisited ? c->m_next : c->m_unvisited);
        c->m_f = c->m_next;
        if (c->mode) {          // the pull kernels wrote the next bitmap and counted it
            c->fb_cur ^= 1;
            c->fb_valid = 1;
            c->queue_stale = 1;
            c->qsize[c->cur ^ 1] = (uint32_t)c->reached_pull;
        } else {
            c->fb_valid = 0;
            c->queue_stale = 0;
        }
        c->cur ^= 1;
        c->level++;
        c->steps++;
        if (c->qsize[c->cur] == 0) c->done = 1;
        if (c->steps > V + 1) {   // cannot happen for a correct run; stop rather than spin
            c->err = 1;
            c->done = 1;
        }
    }
    if (use_cond) cudaGraphSetConditional(h, c->done ? 0u : 1u);
}

// ------------------------------------------------------------------ host --
int traversal_workspace(olv_graph *g, bool pieces) {
    Workspace &w = g->ws;
    const size_t V = g->V;
    OLV_TRY(w.q0.ensure(V * 4 + 16));
    OLV_TRY(w.q1.ensure(V * 4 + 16));
    OLV_TRY(w.ctl.ensure(sizeof(TravCtl)));
    OLV_TRY(w.fbits.ensure(2 * (((size_t)V + 31) / 32 + 8) * 4));
    if (pieces) {
        const uint64_t np = g->E / g->tune.piece + g->E / g->tune.hub_degree + 16;
        OLV_TRY(w.pieces.ensure(np * sizeof(uint2)));
    }
    if (g->persist_blocks == 0) {
        int per_sm = 0;
        OLV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, k_advance_chunks<BfsPushOp>, kBlock, 0));
        if (per_sm < 1) per_sm = 1;
        g->persist_blocks = per_sm * g->num_sms;
    }
    return OLV_OK;
}

__global__ void k_indeg_keys(const uint32_t *__restrict__ colptr, uint32_t V,
                             uint32_t *__restrict__ key, uint32_t *__restrict__ val,
                             unsigned int *__restrict__ counts) {
    unsigned heavy = 0, light = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t d = colptr[v + 1] - colptr[v];
        key[v] = d;
        val[v] = (uint32_t)v;
        heavy += d > kPullHeavy;
        light += d > 0 && d <= kPullHeavy;
    }
    if (heavy) atomicAdd(&counts[0], heavy);
    if (light) atomicAdd(&counts[1], light);
}

// key = (dst << 32) | ~outdeg(src) for every CSC entry: sorting by it orders
// each vertex's in-edges from the highest out-degree source down.
__global__ void k_pull_keys(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowidx,
                            const uint32_t *__restrict__ rowptr, uint32_t V,
                            unsigned long long *__restrict__ key) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = warp; v < V; v += nwarps) {
        const uint32_t b = colptr[v], e = colptr[v + 1];
        for (uint32_t i = b + lane; i < e; i += 32) {
            const uint32_t u = rowidx[i];
            const uint32_t d = rowptr[u + 1] - rowptr[u];
            key[i] = ((unsigned long long)v << 32) | (0xffffffffu - d);
        }
    }
}

// Vertices with in-edges, sorted by in-degree (descending, ties by id), split
// into heavy and light lists for the pull kernel, and the in-edge lists
// reordered so each vertex first probes its highest out-degree in-neighbours
// (the ones a BFS reaches first); built once per graph.
int bfs_pull_lists(olv_graph *g) {
    Workspace &w = g->ws;
    if (w.order.p) return OLV_OK;
    const uint32_t V = g->V;
    cudaStream_t s = g->stream;
    DevBuf key, val, key2, temp, cnt;
    OLV_TRY(key.ensure((size_t)V * 4));
    OLV_TRY(val.ensure((size_t)V * 4));
    OLV_TRY(key2.ensure((size_t)V * 4));
    OLV_TRY(cnt.ensure(16));
    OLV_TRY(w.order.ensure((size_t)V * 4 + 16));
    OLV_CUDA(cudaMemsetAsync(cnt.p, 0, 16, s));
    k_indeg_keys<<<g->num_sms * 8, kBlock, 0, s>>>(g->colptr.as<uint32_t>(), V, key.as<uint32_t>(),
                                                  val.as<uint32_t>(), cnt.as<unsigned int>());
    size_t tb = 0;
    OLV_CUDA(cub::DeviceRadixSort::SortPairsDescending(
        nullptr, tb, (const uint32_t *)nullptr, (uint32_t *)nullptr, (const uint32_t *)nullptr,
        (uint32_t *)nullptr, (int64_t)V, 0, 32, s));
    OLV_TRY(temp.ensure(tb));
    OLV_CUDA(cub::DeviceRadixSort::SortPairsDescending(
        temp.p, tb, key.as<uint32_t>(), key2.as<uint32_t>(), val.as<uint32_t>(),
        w.order.as<uint32_t>(), (int64_t)V, 0, 32, s));
    unsigned int h[2];
    OLV_CUDA(cudaMemcpyAsync(h, cnt.p, 8, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    w.n_heavy = h[0];
    w.n_light = h[1];
    OLV_TRY(w.cand.ensure((size_t)V * 4 + 16));   // pull overflow list
    key.release();
    val.release();
    key2.release();
    temp.release();
    // in-edges by source out-degree, stable (ties keep ascending source ids)
    const uint64_t E = g->E;
    OLV_TRY(w.pull_idx.ensure(E * 4 + 16));
    if (E) {
        DevBuf k0, k1;
        OLV_TRY(k0.ensure(E * 8));
        OLV_TRY(k1.ensure(E * 8));
        k_pull_keys<<<g->num_sms * 16, kBlock, 0, s>>>(g->colptr.as<uint32_t>(),
                                                      g->rowidx.as<uint32_t>(),
                                                      g->rowptr.as<uint32_t>(), V,
                                                      k0.as<unsigned long long>());
        size_t tb2 = 0;
        OLV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb2, (const unsigned long long *)nullptr,
                                                 (unsigned long long *)nullptr,
                                                 (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                                 (int64_t)E, 0, 64, s));
        OLV_TRY(temp.ensure(tb2));
        OLV_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb2, k0.as<unsigned long long>(),
                                                 k1.as<unsigned long long>(),
                                                 g->rowidx.as<uint32_t>(),
                                                 w.pull_idx.as<uint32_t>(), (int64_t)E, 0, 64, s));
        OLV_CUDA(cudaStreamSynchronize(s));
    }
    return OLV_OK;
}

static AdvanceArgs bfs_adv_args(olv_graph *g) {
    AdvanceArgs a;
    a.rbeg = g->rowptr.as<uint32_t>();
    a.rend = g->rowptr.as<uint32_t>() + 1;
    a.col = g->col.as<uint32_t>();
    a.ctl = g->ws.ctl.as<TravCtl>();
    a.q0 = g->ws.q0.as<uint32_t>();
    a.q1 = g->ws.q1.as<uint32_t>();
    a.far0 = a.far1 = nullptr;
    a.pieces = g->ws.pieces.as<uint2>();
    a.hub_degree = g->tune.hub_degree;
    a.piece = g->tune.piece;
    a.want_mode = 0;
    a.rbeg2 = a.rend2 = nullptr;
    a.want_mode2 = 0xffffffffu;
    return a;
}

// One superstep's kernel chain, either launched on a stream or added to a graph.
template <class Sink>
static int bfs_superstep(olv_graph *g, Sink &&sink, cudaGraphConditionalHandle h, int use_cond) {
    TravCtl *ctl = g->ws.ctl.as<TravCtl>();
    uint32_t V = g->V;
    float alpha = g->tune.alpha, beta = g->tune.beta;
    AdvanceArgs a = bfs_adv_args(g);
    BfsPushOp op = {};
    op.rowptr = g->rowptr.as<uint32_t>();
    const uint32_t *colptr = g->colptr.as<uint32_t>();
    const uint32_t *rowptr = g->rowptr.as<uint32_t>();
    uint32_t *q0 = a.q0, *q1 = a.q1;
    const int nb = g->persist_blocks;
    PullLists pl;
    pl.V = V;
    pl.pidx = g->ws.pull_idx.as<uint32_t>();
    pl.order = g->ws.order.as<uint32_t>();
    pl.n_heavy = g->ws.n_heavy;
    pl.n_light = g->ws.n_light;
    pl.cand = g->ws.cand.as<uint32_t>();
    pl.words = ((uint32_t)V + 31) / 32 + 8;
    pl.fb0 = g->ws.fbits.as<uint32_t>();
    pl.fb1 = pl.fb0 + pl.words;
    void *a_begin[] = {&ctl, &V, &alpha, &beta};
    OLV_TRY(sink((const void *)k_bfs_begin, dim3(1), dim3(1), a_begin));
    void *a_fq[] = {&ctl, &q0, &q1, &pl};
    OLV_TRY(sink((const void *)k_bfs_fb_to_queue, dim3(nb), dim3(kBlock), a_fq));
    void *a_adv[] = {&a, &op};
    OLV_TRY(sink((const void *)k_advance_chunks<BfsPushOp>, dim3(nb), dim3(kBlock), a_adv));
    OLV_TRY(sink((const void *)k_advance_pieces<BfsPushOp>, dim3(nb), dim3(kBlock), a_adv));
    void *a_prep[] = {&V, &ctl, &pl};
    OLV_TRY(sink((const void *)k_bfs_pull_prep, dim3(nb), dim3(kBlock), a_prep));
    void *a_pull[] = {&colptr, &rowptr, &ctl, &q0, &q1, &pl};
    OLV_TRY(sink((const void *)k_bfs_pull, dim3(nb), dim3(kBlock), a_pull));
    OLV_TRY(sink((const void *)k_bfs_pull_overflow, dim3(nb), dim3(kBlock), a_pull));
    void *a_end[] = {&ctl, &h, &use_cond, &V};
    OLV_TRY(sink((const void *)k_bfs_end, dim3(1), dim3(1), a_end));
    return OLV_OK;
}

static int bfs_graph(olv_graph *g) {
    if (g->bfs_graph && g->bfs_graph->ready) return OLV_OK;
    if (!g->bfs_graph) g->bfs_graph = new WhileGraph();
    WhileGraph &wg = *g->bfs_graph;
    OLV_TRY(wg.begin());
    auto sink = [&](const void *f, dim3 gr, dim3 bl, void **args) { return wg.add(f, gr, bl, args); };
    OLV_TRY(bfs_superstep(g, sink, wg.handle, 1));
    return wg.finish();
}

int run_bfs_device(olv_graph *g, uint32_t src, int32_t *level_dev) {
    cudaStream_t s = g->stream;
    TravCtl *ctl = g->ws.ctl.as<TravCtl>();
    const int fill_blocks = g->num_sms * 8;
    k_fill_i32<<<fill_blocks, kBlock, 0, s>>>(level_dev, g->V, kInf);
    k_bfs_init<<<1, 1, 0, s>>>(ctl, level_dev, g->ws.q0.as<uint32_t>(), g->rowptr.as<uint32_t>(),
                               src, (unsigned long long)g->E);
    OLV_CUDA(cudaGetLastError());
    if (g->tune.use_graphs) {
        int r = bfs_graph(g);
        if (r == OLV_OK) return g->bfs_graph->launch(s);
        g->tune.use_graphs = 0;   // conditional graphs unavailable: host loop below
    }
    auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
        OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
        return OLV_OK;
    };
    for (;;) {
        for (int i = 0; i < g->tune.levels_per_sync; i++) OLV_TRY(bfs_superstep(g, launch, 0, 0));
        OLV_CUDA(cudaMemcpyAsync(g->host_ctl, ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, s));
        OLV_CUDA(cudaStreamSynchronize(s));
        if (g->host_ctl->done) break;
    }
    return OLV_OK;
}

}  // namespace olv

using namespace olv;

extern "C" int olv_bfs(olv_graph *g, uint32_t src, int32_t *level_out, olv_stats *st) {
    OLV_CHECK_ARG(g && level_out, "olv_bfs: null pointer");
    OLV_CHECK_ARG(src < g->V, "olv_bfs: source %u out of range (V=%u)", src, g->V);
    OLV_TRY(traversal_workspace(g, true));
    OLV_TRY(bfs_pull_lists(g));
    const bool dev_out = is_device_ptr(level_out);
    if (!dev_out) OLV_TRY(g->ws.level.ensure((size_t)g->V * 4 + 16));
    int32_t *level = dev_out ? level_out : g->ws.level.as<int32_t>();
    cudaStream_t s = g->stream;
    OLV_CUDA(cudaEventRecord(g->ev0, s));
    OLV_TRY(run_bfs_device(g, src, level));
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    OLV_CUDA(cudaMemcpyAsync(g->host_ctl, g->ws.ctl.p, sizeof(TravCtl), cudaMemcpyDeviceToHost, s));
    if (!dev_out)
        OLV_CUDA(cudaMemcpyAsync(level_out, level, (size_t)g->V * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    const TravCtl &h = *g->host_ctl;
    if (h.err) {
        set_error("olv_bfs: device-side check failed (code %u)", h.err);
        return OLV_ERR_STATE;
    }
    if (st) {
        float ms = 0;
        OLV_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        st->iterations = h.steps;
        st->pull_steps = h.pull_steps;
        st->vertices_reached = h.reached;
        st->edges_traversed = h.edges_traversed;
        st->edges_relaxed = h.edges_traversed;
        st->residual = 0;
        st->device_ms = ms;
    }
    return OLV_OK;
}
