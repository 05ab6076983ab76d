// Multi-source BFS: up to 64 sources advanced together with one uint64 mask
// per vertex (bit s = source s).  No reference counterpart; each source's
// levels equal a plain BFS from it (testBFS.cu:42-87 semantics, int32 levels,
// 0x7fffffff unreached).
//
// Per vertex: visit (sources that reached it), cur (sources whose frontier
// holds it this level), next (sources reaching it next level).  A level is
//   push  (few active vertices): for each active u and out-edge u->v,
//         atomicOr(next[v], cur[u] & ~visit[v])   -- the shared chunk/piece
//         advance of olv_advance.cuh with a 64-bit source value (in the first
//         two levels without the visit gather: apply drops known bits);
//   pull  (large frontier): each vertex with unvisited bits ORs cur[] over its
//         in-edges, stopping once every missing source is found;
//   apply, dense: new = next & ~visit; visit |= new; the new-bit mask of
//         level L+1 is written to slot L+1 of a per-level mask store, and
//         that slot is the next level's cur (no separate cur array is read or
//         cleared); levels past the store use two spare cur arrays and write
//         their pairs straight into the output; vertices with new bits form
//         the next active queue;
//   apply, sparse (a small push level on a shrinking frontier): the push
//         lists the vertices it touches and only they are visited; their
//         levels go straight into the output and every later level is
//         written the same way (the store is not read past that level).
// A final pass turns the stored masks into the [n][V] int32 output, one
// thread per four vertices, so each source's row goes out in 16-byte stores
// and every output element is written once.  Levels run in a CUDA graph as
// for BFS.
#include <string.h>

#include <vector>

#include "olive_b200/olv_advance.cuh"
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"

namespace olv {

int traversal_workspace(olv_graph *g, bool pieces);
int bfs_pull_lists(olv_graph *g);

constexpr uint32_t kMsHeavy = 128;     // in-degree above which pieces are used (same split as BFS)
constexpr uint32_t kMsPiece = 2048;    // in-edges per heavy piece
constexpr uint32_t kMsSlots = 16;      // levels whose new-bit masks are stored (0 .. 15)

struct MsState {
    DevBuf masks;     // visit | next | cur A | cur B, V words each (A, B: levels >= kMsSlots)
    DevBuf store;     // new-bit masks of levels 0 .. kMsSlots-1, V words each
    DevBuf touched;   // vertices first touched by a tracked push level
    DevBuf srcs;
    DevBuf pieces;    // (vertex, first in-edge, end) of heavy vertices' in-edge pieces
    uint32_t npieces = 0;
    WhileGraph graph;
    int32_t *graph_levels = nullptr;
    uint32_t graph_n = 0;
    ~MsState() {
        masks.release();
        store.release();
        touched.release();
        srcs.release();
        pieces.release();
        graph.destroy();
    }
};

// The frontier mask of level L: slot L of the mask store, or one of two
// spare arrays for the levels past the store.
struct MsCur {
    unsigned long long *store, *cx0, *cx1;
    uint32_t V;
    __device__ __forceinline__ unsigned long long *at(uint32_t L) const {
        return L < kMsSlots ? store + (uint64_t)L * V : ((L & 1) ? cx1 : cx0);
    }
};

struct MsPushOp {
    using SV = unsigned long long;
    static constexpr int kMinBlocks = 1;   // CTAs per SM the advance must fit
    static constexpr bool kHasFar = false;
    static constexpr bool kPacked = false;
    MsCur cm;
    const unsigned long long *cur;
    const unsigned long long *visit;
    unsigned long long *next;
    uint32_t *touched;          // first-touched vertices of a tracked level
    uint32_t *ntouched;
    uint32_t track;
    uint32_t filter;            // drop source bits the target already has
    struct Pre {
        unsigned long long bits;
    };
    __device__ __forceinline__ void begin(TravCtl *c) {
        cur = cm.at(c->level);
        track = c->ms_track;
        ntouched = &c->ms_touched;
        // in the first two levels almost no target has been visited yet:
        // skip the visit gather per edge and let apply drop known bits
        filter = c->level >= 2;
    }
    __device__ __forceinline__ SV src_value(uint32_t u) const { return cur[u]; }
    __device__ __forceinline__ bool on_input(uint32_t) const { return true; }
    __device__ __forceinline__ Pre prepare(SV sv, uint32_t, uint32_t v) const {
        return Pre{filter ? sv & ~__ldg(&visit[v]) : sv};
    }
    // OR the source bits into next[v]; on a tracked level, also list every v
    // whose next mask was zero before (once per vertex and level), with one
    // list atomic per warp.  All 32 lanes call it.
    template <int N>
    __device__ __forceinline__ void apply_n(const Pre (&p)[N], const uint32_t (&v)[N],
                                            int (&act)[N]) {
        if (!track) {
#pragma unroll
            for (int j = 0; j < N; j++) {
                if (act[j] && p[j].bits) atomicOr(&next[v[j]], p[j].bits);
                act[j] = 0;
            }
            return;
        }
        bool first[N];
        uint32_t cnt = 0;
#pragma unroll
        for (int j = 0; j < N; j++) {
            first[j] = false;
            if (act[j] && p[j].bits) first[j] = atomicOr(&next[v[j]], p[j].bits) == 0ULL;
            cnt += first[j];
            act[j] = 0;
        }
        const uint32_t lane = lane_id();
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        if (!total) return;
        uint32_t base = 0;
        if (lane == 31) base = atomicAdd(ntouched, total);
        base = __shfl_sync(0xffffffffu, base, 31) + incl - cnt;
#pragma unroll
        for (int j = 0; j < N; j++)
            if (first[j]) touched[base++] = v[j];
    }
    __device__ __forceinline__ void on_push(bool, uint32_t) {}
    __device__ __forceinline__ void flush(unsigned long long) {}
};

// levels[s][v] = value for every set bit s of bits.  All 32 lanes call it with
// consecutive v: the loop runs over the bits set in any lane, so each store
// instruction writes one row s at consecutive columns (coalesced).
__device__ __forceinline__ void write_levels_warp(int32_t *levels, uint64_t V, uint32_t v,
                                                  unsigned long long bits, int32_t value) {
    unsigned long long any = bits;
#pragma unroll
    for (int o = 16; o; o >>= 1) any |= __shfl_xor_sync(0xffffffffu, any, o);
    while (any) {
        const int s = __ffsll((long long)any) - 1;
        any &= any - 1;
        if ((bits >> s) & 1ULL) levels[(uint64_t)s * V + v] = value;
    }
}

__device__ void ms_begin(TravCtl *c, unsigned long long E, float alpha);

__global__ void k_ms_init(TravCtl *c, int32_t *levels, const uint32_t *srcs, int n, uint32_t V,
                          const uint32_t *rowptr, unsigned long long *visit, uint32_t *q0,
                          unsigned long long *store0, unsigned long long E, float alpha) {
    __shared__ unsigned long long s_edges;
    if (threadIdx.x == 0) {
        TravCtl t = {};
        t.vdata = levels;
        t.ms_sparse_from = 0xffffffffu;
        t.ms_cur_dense = 1;                  // slot 0 is cleared and holds the sources
        t.ms_new_prev = (unsigned long long)n;   // level 0: the sources
        t.ms_new_prev2 = 0;
        *c = t;
        s_edges = 0;
    }
    __syncthreads();
    if ((int)threadIdx.x < n) {
        const uint32_t u = srcs[threadIdx.x];
        const unsigned long long bit = 1ULL << threadIdx.x;
        const unsigned long long old = atomicOr(&store0[u], bit);   // level 0 = cur of level 0
        atomicOr(&visit[u], bit);
        const uint32_t d = rowptr[u + 1] - rowptr[u];
        atomicAdd(&s_edges, (unsigned long long)d);
        if (old == 0) {
            const uint32_t pos = atomicAdd(&c->qsize[0], 1u);
            q0[pos] = u;
            atomicAdd(&c->m_f, (unsigned long long)d);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        c->edges_traversed = s_edges;
        ms_begin(c, E, alpha);   // the first superstep's mode
    }
}

// Mode and counters of the next superstep (called by k_ms_init and k_ms_end).
__device__ void ms_begin(TravCtl *c, unsigned long long E, float alpha) {
    if (c->done) return;
    if (c->qsize[c->cur] == 0) {
        c->done = 1;
        return;
    }
    // after a sparse level the frontier array is valid only at queued
    // vertices, which a push reads and a pull would not: push
    c->mode = (c->ms_cur_dense && (double)c->m_f * alpha > (double)E) ? 1u : 0u;
    // a push on a shrinking frontier lists the vertices it touches, so that a
    // small level can be applied sparsely
    c->ms_track = c->mode == 0 && c->ms_new_prev < c->ms_new_prev2;
    c->ms_touched = 0;
    c->qsize[c->cur ^ 1] = 0;
    c->npieces = 0;
    c->m_next = 0;
    c->reached_pull = 0;
}

// A tracked push level that touched at most V/64 vertices is applied
// sparsely: only its touched vertices are visited, their new bits become the
// next frontier at those vertices only, and their levels are written
// straight into the output (no store slot for this or any later level).
__device__ __forceinline__ bool ms_sparse_level(const TravCtl *c, uint32_t V) {
    return c->ms_track && c->ms_touched <= V / 64;
}

constexpr int kMsParents = 4;
#ifndef OLV_MS_BLOCKS
#define OLV_MS_BLOCKS 2
#endif
constexpr int kMsBlocks = OLV_MS_BLOCKS;   // 16-byte in-edge blocks per light-vertex round

// Pull.  Heavy vertices' in-edges come as pieces of kMsPiece edges, one warp
// per piece, ORed into next[v] with atomicOr (OR is order-free).  Light
// vertices (in-degree 1..kMsHeavy) are scanned by one thread each over
// consecutive ids, eight in-edges per round from two 16-byte index loads.
// Both stop once every missing source is found.
__global__ void __launch_bounds__(kBlock)
k_ms_pull(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowidx, uint32_t V,
          unsigned long long srcmask, const TravCtl *c, const unsigned long long *__restrict__ visit,
          MsCur cm, unsigned long long *__restrict__ next, const uint4 *__restrict__ pieces,
          uint32_t npieces) {
    if (c->done || c->mode != 1) return;
    const unsigned long long *__restrict__ cur = cm.at(c->level);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = gwarp; p < npieces; p += nwarps) {
        const uint4 pc = pieces[p];
        const uint32_t v = pc.x;
        const unsigned long long todo = ~visit[v] & srcmask;
        if (!todo) continue;
        unsigned long long acc = 0;
        for (uint32_t base = pc.y; base < pc.z; base += 32 * kMsParents) {
#pragma unroll
            for (int j = 0; j < kMsParents; j++) {
                const uint32_t i = base + j * 32 + lane;
                if (i < pc.z) acc |= __ldg(&cur[__ldg(&rowidx[i])]);
            }
            unsigned long long all = acc;
#pragma unroll
            for (int o = 16; o; o >>= 1) all |= __shfl_xor_sync(0xffffffffu, all, o);
            if ((all & todo) == todo) break;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0 && (acc & todo)) atomicOr(&next[v], acc & todo);
    }
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = __ldg(&colptr[v]), e = __ldg(&colptr[v + 1]);
        if (e - b > kMsHeavy || e == b) continue;
        const unsigned long long todo = ~visit[v] & srcmask;
        if (!todo) continue;
        // in-edges read as aligned 16-byte blocks (the index array is padded
        // to a multiple of 4 entries), kMsBlocks blocks per round; entries
        // outside [b, e) are skipped
        unsigned long long acc = 0;
        for (uint32_t blk = b & ~3u; blk < e; blk += 4 * kMsBlocks) {
            uint32_t u[4 * kMsBlocks];
#pragma unroll
            for (int k = 0; k < kMsBlocks; k++) {
                const uint4 x = (k == 0 || blk + 4 * k < e)
                                    ? __ldg(reinterpret_cast<const uint4 *>(rowidx + blk + 4 * k))
                                    : make_uint4(0, 0, 0, 0);
                u[4 * k] = x.x;
                u[4 * k + 1] = x.y;
                u[4 * k + 2] = x.z;
                u[4 * k + 3] = x.w;
            }
#pragma unroll
            for (int j = 0; j < 4 * kMsBlocks; j++)
                if (blk + j >= b && blk + j < e) acc |= __ldg(&cur[u[j]]);
            if ((acc & todo) == todo) break;
        }
        if (acc & todo) atomicOr(&next[v], acc & todo);
    }
}

__global__ void __launch_bounds__(kBlock)
k_ms_apply(uint32_t V, TravCtl *c, const uint32_t *__restrict__ rowptr,
           unsigned long long *__restrict__ visit, MsCur cm,
           unsigned long long *__restrict__ next, uint32_t *q0, uint32_t *q1,
           const uint32_t *__restrict__ touched) {
    if (c->done) return;
    int32_t *levels = static_cast<int32_t *>(c->vdata);
    // vertices with new bits form the next level's queue (per-warp staging)
    uint32_t *q = c->cur ? q0 : q1;
    uint32_t *qsize = &c->qsize[c->cur ^ 1];
    __shared__ uint32_t s_q[kBlock / 32][kWarpStage];
    __shared__ uint32_t s_n[kBlock / 32], s_lim[kBlock / 32];
    const uint32_t wl = threadIdx.x >> 5;
    if (lane_id() == 0) {
        s_n[wl] = 0;
        s_lim[wl] = kWarpStage;
    }
    __syncwarp();
    const int32_t lv = (int32_t)c->level + 1;
    // the next level's cur: slot lv of the mask store, or a spare array (and
    // direct writes of the level into the output) past the store
    unsigned long long *__restrict__ ncur = cm.at((uint32_t)lv);
    const bool past = (uint32_t)lv >= kMsSlots || (uint32_t)lv >= c->ms_sparse_from;
    unsigned long long m_next = 0, traversed = 0, nact = 0;
    if (ms_sparse_level(c, V)) {
        // sparse: one thread per touched vertex (the vertices whose next mask
        // the push made nonzero); new bits join visit, become the next
        // frontier at that vertex, and their level goes straight into each
        // source's row
        const uint32_t nt = c->ms_touched;
        const uint32_t sstride = gridDim.x * kBlock;
        for (uint32_t b = blockIdx.x * kBlock; b < nt; b += sstride) {   // warp-uniform
            const uint32_t i = b + threadIdx.x;
            bool act = false;
            uint32_t v = 0;
            if (i < nt) {
                v = touched[i];
                const unsigned long long nx = next[v];
                next[v] = 0;
                const unsigned long long vis = visit[v];
                const unsigned long long nw = nx & ~vis;
                if (nw) {
                    visit[v] = vis | nw;
                    ncur[v] = nw;
                    const uint32_t d = __ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]);
                    m_next += d;
                    traversed += (unsigned long long)d * __popcll(nw);
                    act = true;
                    for (unsigned long long bb = nw; bb; bb &= bb - 1)
                        levels[(uint64_t)(__ffsll((long long)bb) - 1) * V + v] = lv;
                }
            }
            nact += act;
            int pa[1] = {act};
            uint32_t pv[1] = {v};
            __syncwarp();
            if (s_n[wl] + 32 > kWarpStage) warp_stage_flush(s_q[wl], &s_n[wl], &s_lim[wl], q, qsize);
            stage_push_n<1>(pa, pv, 1, s_q[wl], &s_n[wl], &s_lim[wl], kWarpStage, q, qsize);
        }
        warp_stage_flush(s_q[wl], &s_n[wl], &s_lim[wl], q, qsize);
        warp_add64(m_next, &c->m_next);
        warp_add64(traversed, &c->edges_traversed);
        warp_add64(nact, &c->reached_pull);
        return;
    }
    // dense: kApply vertices per thread, strided by the grid so each load stays
    // coalesced; all their next loads are issued before any is used
    constexpr int kApply = 4;
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < V; base += stride * kApply) {
        unsigned long long nx[kApply];
#pragma unroll
        for (int k = 0; k < kApply; k++) {
            const uint64_t v = base + k * stride + threadIdx.x;
            nx[k] = v < V ? next[v] : 0ULL;
        }
#pragma unroll
        for (int k = 0; k < kApply; k++) {
            const uint64_t v = base + k * stride + threadIdx.x;
            unsigned long long nw = 0;
            bool act = false;
            if (v < V) {
                if (nx[k]) {
                    const unsigned long long vis = visit[v];
                    nw = nx[k] & ~vis;
                    next[v] = 0;
                    if (nw) {
                        visit[v] = vis | nw;
                        const uint32_t d = __ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]);
                        m_next += d;
                        traversed += (unsigned long long)d * __popcll(nw);
                        act = true;
                    }
                }
                ncur[v] = nw;
            }
            // warp-uniform: base, k and stride are the same for the whole warp
            if (past && base + k * stride < V) write_levels_warp(levels, V, (uint32_t)v, nw, lv);
            nact += act;
            int pa[1] = {act};
            uint32_t pv[1] = {(uint32_t)v};
            __syncwarp();
            if (s_n[wl] + 32 > kWarpStage) warp_stage_flush(s_q[wl], &s_n[wl], &s_lim[wl], q, qsize);
            stage_push_n<1>(pa, pv, 1, s_q[wl], &s_n[wl], &s_lim[wl], kWarpStage, q, qsize);
        }
    }
    warp_stage_flush(s_q[wl], &s_n[wl], &s_lim[wl], q, qsize);
    warp_add64(m_next, &c->m_next);
    warp_add64(traversed, &c->edges_traversed);
    warp_add64(nact, &c->reached_pull);
}

__global__ void k_ms_end(TravCtl *c, cudaGraphConditionalHandle h, int use_cond, uint32_t V,
                         unsigned long long E, float alpha) {
    if (!c->done) {
        if (c->mode) c->pull_steps++;
        if (ms_sparse_level(c, V)) {
            c->ms_cur_dense = 0;
            if (c->ms_sparse_from == 0xffffffffu) c->ms_sparse_from = c->level + 1;
        } else {
            c->ms_cur_dense = 1;
        }
        c->ms_new_prev2 = c->ms_new_prev;
        c->ms_new_prev = c->reached_pull;
        c->m_f = c->m_next;
        c->cur ^= 1;
        c->level++;
        c->steps++;
        if (c->qsize[c->cur] == 0) c->done = 1;
        if (c->steps > V + 1) {
            c->err = 1;
            c->done = 1;
        }
        ms_begin(c, E, alpha);   // the next superstep's mode and counters
    }
    if (use_cond) cudaGraphSetConditional(h, c->done ? 0u : 1u);
}

// The [n][V] output from the stored level masks.  Each source's bit is set
// in at most one slot, so OR-ing the slot masks by the bits of the slot index
// gives four masks whose bit q spells source q's level (levels 0..15) with no
// per-bit loop.  A lane holds one vertex; for each source q it writes
// 0x7fffffff (never reached), the stored level, or nothing (a level past the
// store, written by apply), and the 32 lanes' stores form one 128-byte line of
// row q.  The masks are kept as 32-bit halves so that every source's bits
// come out with constant shifts (the source loop is unrolled).  Also counts
// the reached pairs.
static_assert(kMsSlots == 16, "four level bits");

// Row q of the output for sources q0 .. q0+31 of one vertex, from 32-bit
// halves of the level-bit masks (b0..b3), the stored-level mask and the
// visit mask.  `out` points at row q0, column v.  For each group of eight
// sources the four planes' bytes are packed into one word W (b3, b2, b1, b0
// from the low byte up); a source's level is then (((W >> j) & 0x01010101)
// * 0x08040201) >> 24: the multiply lines the four bits up at bits 24..27
// (8 b3 + 4 b2 + 2 b1 + b0), with no carries since no two partial products
// share a bit.
template <int Q0>
__device__ __forceinline__ void ms_write_half(int32_t *out, uint64_t V, int n, uint32_t b0,
                                              uint32_t b1, uint32_t b2, uint32_t b3, uint32_t any,
                                              uint32_t vis) {
#pragma unroll
    for (int m = 0; m < 4; m++) {
        if (Q0 + 8 * m >= n) break;
        const uint32_t sel = (uint32_t)m | ((4u + m) << 4);
        const uint32_t lo = __byte_perm(b3, b2, sel);   // [b3.m, b2.m, -, -]
        const uint32_t hi = __byte_perm(b1, b0, sel);   // [b1.m, b0.m, -, -]
        const uint32_t W = __byte_perm(lo, hi, 0x5410);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (Q0 + 8 * m + j >= n) break;
            const int32_t lvl = (int32_t)((((W >> j) & 0x01010101u) * 0x08040201u) >> 24);
            const bool reached = (vis >> (8 * m + j)) & 1u;
            const bool stored = (any >> (8 * m + j)) & 1u;
            if (!reached || stored) __stcs(out, reached ? lvl : kInf);
            out += V;
        }
    }
}

__global__ void __launch_bounds__(kBlock, 4)
k_ms_levels(uint32_t V, int n, unsigned long long srcmask, TravCtl *c,
            const unsigned long long *__restrict__ visit,
            const unsigned long long *__restrict__ store) {
    int32_t *levels = static_cast<int32_t *>(c->vdata);
    // slots 0 .. level-1: the run ended because level `level` found no new
    // vertex, so its slot is all zeros and is not read
    uint32_t nst = c->level < kMsSlots ? c->level : kMsSlots;
    if (nst > c->ms_sparse_from) nst = c->ms_sparse_from;   // later levels were written directly
    unsigned long long reached = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)kBlock + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * kBlock) {
        const unsigned long long vis = visit[v] & srcmask;
        reached += __popcll(vis);
        unsigned long long m[kMsSlots];
#pragma unroll
        for (uint32_t L = 0; L < kMsSlots; L++)
            m[L] = L < nst ? __ldcs(&store[(uint64_t)L * V + v]) : 0ULL;
        unsigned long long b0 = 0, b1 = 0, b2 = 0, b3 = 0, any = 0;
#pragma unroll
        for (uint32_t L = 0; L < kMsSlots; L++) {
            any |= m[L];
            if (L & 1) b0 |= m[L];
            if (L & 2) b1 |= m[L];
            if (L & 4) b2 |= m[L];
            if (L & 8) b3 |= m[L];
        }
        int32_t *out = levels + v;
        ms_write_half<0>(out, V, n, (uint32_t)b0, (uint32_t)b1, (uint32_t)b2, (uint32_t)b3,
                         (uint32_t)any, (uint32_t)vis);
        if (n > 32)
            ms_write_half<32>(out + 32 * (uint64_t)V, V, n, (uint32_t)(b0 >> 32),
                              (uint32_t)(b1 >> 32), (uint32_t)(b2 >> 32), (uint32_t)(b3 >> 32),
                              (uint32_t)(any >> 32), (uint32_t)(vis >> 32));
    }
    warp_add64(reached, &c->reached);
}

// The same output with one thread per four consecutive vertices, each row's
// four levels written as one 16-byte store (a warp writes 512 contiguous
// bytes of a row).  Needs V % 4 == 0 and a 16-byte aligned output.
__device__ __forceinline__ uint32_t ms_pack_planes(uint32_t b0, uint32_t b1, uint32_t b2,
                                                   uint32_t b3, uint32_t m) {
    const uint32_t sel = m | ((4u + m) << 4);
    return __byte_perm(__byte_perm(b3, b2, sel), __byte_perm(b1, b0, sel), 0x5410);
}

template <int Q0>
__device__ __forceinline__ void ms_write_half4(int32_t *out, uint64_t V, int n,
                                               const uint32_t (&b0)[4], const uint32_t (&b1)[4],
                                               const uint32_t (&b2)[4], const uint32_t (&b3)[4],
                                               const uint32_t (&any)[4], const uint32_t (&vis)[4]) {
#pragma unroll
    for (int m = 0; m < 4; m++) {
        if (Q0 + 8 * m >= n) break;
        uint32_t W[4];
#pragma unroll
        for (int k = 0; k < 4; k++) W[k] = ms_pack_planes(b0[k], b1[k], b2[k], b3[k], m);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (Q0 + 8 * m + j >= n) break;
            int32_t val[4];
            bool skip = false;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int32_t lvl = (int32_t)((((W[k] >> j) & 0x01010101u) * 0x08040201u) >> 24);
                const bool reached = (vis[k] >> (8 * m + j)) & 1u;
                const bool stored = (any[k] >> (8 * m + j)) & 1u;
                val[k] = reached ? lvl : kInf;
                skip |= reached && !stored;
            }
            if (!skip) {
                __stcs(reinterpret_cast<int4 *>(out), make_int4(val[0], val[1], val[2], val[3]));
            } else {   // a level past the store, written by apply: leave it
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const bool reached = (vis[k] >> (8 * m + j)) & 1u;
                    const bool stored = (any[k] >> (8 * m + j)) & 1u;
                    if (!reached || stored) __stcs(out + k, val[k]);
                }
            }
            out += V;
        }
    }
}

__global__ void __launch_bounds__(kBlock, 3)
k_ms_levels4(uint32_t V, int n, unsigned long long srcmask, TravCtl *c,
             const unsigned long long *__restrict__ visit,
             const unsigned long long *__restrict__ store) {
    int32_t *levels = static_cast<int32_t *>(c->vdata);
    // slots 0 .. level-1: the run ended because level `level` found no new
    // vertex, so its slot is all zeros and is not read
    uint32_t nst = c->level < kMsSlots ? c->level : kMsSlots;
    if (nst > c->ms_sparse_from) nst = c->ms_sparse_from;   // later levels were written directly
    unsigned long long reached = 0;
    const uint64_t nq = V / 4;
    for (uint64_t t = blockIdx.x * (uint64_t)kBlock + threadIdx.x; t < nq;
         t += (uint64_t)gridDim.x * kBlock) {
        const uint64_t v0 = 4 * t;
        const ulonglong2 va = __ldcs(reinterpret_cast<const ulonglong2 *>(visit + v0));
        const ulonglong2 vb = __ldcs(reinterpret_cast<const ulonglong2 *>(visit + v0 + 2));
        unsigned long long vis[4] = {va.x & srcmask, va.y & srcmask, vb.x & srcmask, vb.y & srcmask};
        unsigned long long B0[4] = {0, 0, 0, 0}, B1[4] = {0, 0, 0, 0}, B2[4] = {0, 0, 0, 0},
                           B3[4] = {0, 0, 0, 0}, AN[4] = {0, 0, 0, 0};
#pragma unroll
        for (uint32_t L = 0; L < kMsSlots; L++) {
            if (L >= nst) break;
            const unsigned long long *sl = store + (uint64_t)L * V + v0;
            const ulonglong2 x = __ldcs(reinterpret_cast<const ulonglong2 *>(sl));
            const ulonglong2 y = __ldcs(reinterpret_cast<const ulonglong2 *>(sl + 2));
            const unsigned long long mk[4] = {x.x, x.y, y.x, y.y};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                AN[k] |= mk[k];
                if (L & 1) B0[k] |= mk[k];
                if (L & 2) B1[k] |= mk[k];
                if (L & 4) B2[k] |= mk[k];
                if (L & 8) B3[k] |= mk[k];
            }
        }
        uint32_t b0[4], b1[4], b2[4], b3[4], an[4], vs[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            reached += __popcll(vis[k]);
            b0[k] = (uint32_t)B0[k];
            b1[k] = (uint32_t)B1[k];
            b2[k] = (uint32_t)B2[k];
            b3[k] = (uint32_t)B3[k];
            an[k] = (uint32_t)AN[k];
            vs[k] = (uint32_t)vis[k];
        }
        int32_t *out = levels + v0;
        ms_write_half4<0>(out, V, n, b0, b1, b2, b3, an, vs);
        if (n > 32) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                b0[k] = (uint32_t)(B0[k] >> 32);
                b1[k] = (uint32_t)(B1[k] >> 32);
                b2[k] = (uint32_t)(B2[k] >> 32);
                b3[k] = (uint32_t)(B3[k] >> 32);
                an[k] = (uint32_t)(AN[k] >> 32);
                vs[k] = (uint32_t)(vis[k] >> 32);
            }
            ms_write_half4<32>(out + 32 * (uint64_t)V, V, n, b0, b1, b2, b3, an, vs);
        }
    }
    warp_add64(reached, &c->reached);
}

// ------------------------------------------------------------------ host --
template <class Sink>
static int ms_superstep(olv_graph *g, MsState &ms, Sink &&sink, cudaGraphConditionalHandle h,
                        int use_cond, unsigned long long srcmask) {
    TravCtl *ctl = g->ws.ctl.as<TravCtl>();
    uint32_t V = g->V;
    unsigned long long E = g->E;
    float alpha = g->tune.ms_alpha;
    unsigned long long *visit = ms.masks.as<unsigned long long>();
    unsigned long long *next = visit + V;
    MsCur cm;
    cm.store = ms.store.as<unsigned long long>();
    cm.cx0 = visit + 2 * (size_t)V;
    cm.cx1 = visit + 3 * (size_t)V;
    cm.V = V;
    AdvanceArgs a;
    a.rbeg = g->rowptr.as<uint32_t>();
    a.rend = g->rowptr.as<uint32_t>() + 1;
    a.col = g->col.as<uint32_t>();
    a.ctl = ctl;
    a.q0 = g->ws.q0.as<uint32_t>();
    a.q1 = g->ws.q1.as<uint32_t>();
    a.far0 = a.far1 = nullptr;
    a.pieces = g->ws.pieces.as<uint2>();
    a.hub_degree = g->tune.hub_degree;
    a.piece = g->tune.piece;
    a.want_mode = 0;
    a.rbeg2 = a.rend2 = nullptr;
    a.want_mode2 = 0xffffffffu;
    MsPushOp op;
    op.cm = cm;
    op.cur = nullptr;
    op.touched = ms.touched.as<uint32_t>();
    op.ntouched = nullptr;
    op.track = 0;
    op.filter = 1;
    op.visit = visit;
    op.next = next;
    const uint32_t *colptr = g->colptr.as<uint32_t>();
    // in-edges ordered by source out-degree: early exits come sooner
    const uint32_t *rowidx = g->ws.pull_idx.p ? g->ws.pull_idx.as<uint32_t>()
                                              : g->rowidx.as<uint32_t>();
    const uint32_t *rowptr = g->rowptr.as<uint32_t>();
    const TravCtl *cctl = ctl;
    const unsigned long long *cvisit = visit;
    uint32_t *q0 = a.q0, *q1 = a.q1;
    int nb = 0;
    OLV_TRY(resident_blocks(g, (const void *)k_advance_chunks<MsPushOp>, &nb));
    void *a_adv[] = {&a, &op};
    OLV_TRY(sink((const void *)k_advance_chunks<MsPushOp>, dim3(nb), dim3(kBlock), a_adv));
    OLV_TRY(sink((const void *)k_advance_pieces<MsPushOp>, dim3(nb), dim3(kBlock), a_adv));
    const uint4 *pcs = ms.pieces.as<uint4>();
    uint32_t npcs = ms.npieces;
    void *a_pull[] = {&colptr, &rowidx, &V, &srcmask, &cctl, &cvisit, &cm, &next, &pcs, &npcs};
    // the pull and apply passes are latency bound: each runs at its own full
    // residency (the advance is held to fewer CTAs by its registers)
    int nb_pull = 0, nb_apply = 0;
    OLV_TRY(resident_blocks(g, (const void *)k_ms_pull, &nb_pull));
    OLV_TRY(resident_blocks(g, (const void *)k_ms_apply, &nb_apply));
    OLV_TRY(sink((const void *)k_ms_pull, dim3(nb_pull), dim3(kBlock), a_pull));
    const uint32_t *touched = ms.touched.as<uint32_t>();
    void *a_apply[] = {&V, &ctl, &rowptr, &visit, &cm, &next, &q0, &q1, &touched};
    OLV_TRY(sink((const void *)k_ms_apply, dim3(nb_apply), dim3(kBlock), a_apply));
    void *a_end[] = {&ctl, &h, &use_cond, &V, &E, &alpha};
    OLV_TRY(sink((const void *)k_ms_end, dim3(1), dim3(1), a_end));
    return OLV_OK;
}

// In-edge pieces of the heavy vertices (in-degree above kMsHeavy), once per graph.
static int ms_pieces(olv_graph *g, MsState &ms) {
    if (ms.pieces.p) return OLV_OK;
    OLV_TRY(bfs_pull_lists(g));
    const uint32_t nh = g->ws.n_heavy;
    std::vector<uint32_t> order(nh), cp((size_t)g->V + 1);
    if (nh)
        OLV_CUDA(cudaMemcpy(order.data(), g->ws.order.p, (size_t)nh * 4, cudaMemcpyDeviceToHost));
    OLV_CUDA(cudaMemcpy(cp.data(), g->colptr.p, ((size_t)g->V + 1) * 4, cudaMemcpyDeviceToHost));
    std::vector<uint4> pcs;
    for (uint32_t i = 0; i < nh; i++) {
        const uint32_t v = order[i], b = cp[v], e = cp[v + 1];
        for (uint32_t x = b; x < e; x += kMsPiece)
            pcs.push_back(make_uint4(v, x, e - x > kMsPiece ? x + kMsPiece : e, 0));
    }
    ms.npieces = (uint32_t)pcs.size();
    OLV_TRY(ms.pieces.ensure(pcs.size() * sizeof(uint4) + 16));
    if (!pcs.empty())
        OLV_CUDA(cudaMemcpy(ms.pieces.p, pcs.data(), pcs.size() * sizeof(uint4),
                            cudaMemcpyHostToDevice));
    return OLV_OK;
}

static MsState *ms_state(olv_graph *g) {
    if (!g->ms_state) g->ms_state = new MsState();
    return static_cast<MsState *>(g->ms_state);
}

void release_ms_state(olv_graph *g) {
    delete static_cast<MsState *>(g->ms_state);
    g->ms_state = nullptr;
}

}  // namespace olv

using namespace olv;

extern "C" int olv_msbfs(olv_graph *g, const uint32_t *srcs, int n, int32_t *levels_out,
                         olv_stats *st) {
    OLV_CHECK_ARG(g && srcs && levels_out, "olv_msbfs: null pointer");
    OLV_CHECK_ARG(n >= 1 && n <= 64, "olv_msbfs: n=%d sources, must be in [1,64]", n);
    const bool dev_src = is_device_ptr(srcs);
    std::vector<uint32_t> hs(n);
    if (dev_src) {
        OLV_CUDA(cudaMemcpy(hs.data(), srcs, n * 4, cudaMemcpyDeviceToHost));
    } else {
        memcpy(hs.data(), srcs, n * 4);
    }
    for (int i = 0; i < n; i++)
        OLV_CHECK_ARG(hs[i] < g->V, "olv_msbfs: source %u out of range (V=%u)", hs[i], g->V);
    OLV_TRY(traversal_workspace(g, true));
    MsState &ms = *ms_state(g);
    OLV_TRY(ms_pieces(g, ms));
    const size_t V = g->V;
    OLV_TRY(ms.masks.ensure(V * 32 + 64));
    OLV_TRY(ms.store.ensure((size_t)kMsSlots * V * 8 + 64));
    OLV_TRY(ms.touched.ensure(V * 4 + 64));
    OLV_TRY(ms.srcs.ensure(64 * 4));
    const bool dev_out = is_device_ptr(levels_out);
    const size_t out_bytes = (size_t)n * V * 4;
    DevBuf tmp_out;
    if (!dev_out) OLV_TRY(tmp_out.ensure(out_bytes));
    int32_t *levels = dev_out ? levels_out : tmp_out.as<int32_t>();
    cudaStream_t s = g->stream;
    const unsigned long long srcmask = n == 64 ? ~0ULL : ((1ULL << n) - 1);
    TravCtl *ctl = g->ws.ctl.as<TravCtl>();
    unsigned long long *visit = ms.masks.as<unsigned long long>();

    OLV_CUDA(cudaEventRecord(g->ev0, s));
    OLV_CUDA(cudaMemcpyAsync(ms.srcs.p, hs.data(), n * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemsetAsync(ms.masks.p, 0, V * 16, s));   // visit, next
    OLV_CUDA(cudaMemsetAsync(ms.store.p, 0, V * 8, s));   // slot 0: the sources
    k_ms_init<<<1, 64, 0, s>>>(ctl, levels, ms.srcs.as<uint32_t>(), n, g->V,
                               g->rowptr.as<uint32_t>(), visit, g->ws.q0.as<uint32_t>(),
                               ms.store.as<unsigned long long>(), (unsigned long long)g->E,
                               g->tune.ms_alpha);
    OLV_CUDA(cudaGetLastError());
    bool launched = false;
    if (g->tune.use_graphs) {
        if (!ms.graph.ready || ms.graph_n != (uint32_t)n) {
            int r = ms.graph.begin();
            auto sink = [&](const void *f, dim3 gr, dim3 bl, void **args) {
                return ms.graph.add(f, gr, bl, args);
            };
            if (r == OLV_OK) r = ms_superstep(g, ms, sink, ms.graph.handle, 1, srcmask);
            if (r == OLV_OK) r = ms.graph.finish();
            if (r != OLV_OK) ms.graph.destroy();
            ms.graph_n = n;
        }
        if (ms.graph.ready) {
            OLV_TRY(ms.graph.launch(s));
            launched = true;
        }
    }
    if (!launched) {
        auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
            OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
            return OLV_OK;
        };
        for (;;) {
            for (int i = 0; i < g->tune.levels_per_sync; i++)
                OLV_TRY(ms_superstep(g, ms, launch, 0, 0, srcmask));
            OLV_CUDA(cudaMemcpyAsync(g->host_ctl, ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, s));
            OLV_CUDA(cudaStreamSynchronize(s));
            if (g->host_ctl->done) break;
        }
    }
    if (g->V % 4 == 0 && ((uintptr_t)levels & 15) == 0) {   // 16-byte rows of four vertices
        int nb4 = 0;
        OLV_TRY(resident_blocks(g, (const void *)k_ms_levels4, &nb4));
        k_ms_levels4<<<nb4, kBlock, 0, s>>>(g->V, n, srcmask, ctl, visit,
                                            ms.store.as<unsigned long long>());
    }
    else {
        k_ms_levels<<<g->num_sms * 8, kBlock, 0, s>>>(g->V, n, srcmask, ctl, visit,
                                                      ms.store.as<unsigned long long>());
    }
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    OLV_CUDA(cudaMemcpyAsync(g->host_ctl, ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, s));
    if (!dev_out) OLV_CUDA(cudaMemcpyAsync(levels_out, levels, out_bytes, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    const TravCtl &h = *g->host_ctl;
    if (h.err) {
        set_error("olv_msbfs: device-side check failed (code %u)", h.err);
        return OLV_ERR_STATE;
    }
    if (st) {
        float ms_ = 0;
        OLV_CUDA(cudaEventElapsedTime(&ms_, g->ev0, g->ev1));
        st->iterations = h.steps;
        st->pull_steps = h.pull_steps;
        st->vertices_reached = h.reached;          // reached (source, vertex) pairs
        st->edges_traversed = h.edges_traversed;   // sum over sources of E_reached
        st->edges_relaxed = h.edges_traversed;
        st->residual = 0;
        st->device_ms = ms_;
    }
    return OLV_OK;
}
