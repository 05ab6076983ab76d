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

#include "olive_b200/olv_advance.cuh"
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"

namespace olv {

struct BfsPushOp {
    using SV = uint32_t;
    static constexpr int kMinBlocks = 1;   // CTAs per SM the advance must fit
    static constexpr bool kHasFar = false;
    static constexpr bool kPacked = false;
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
    __device__ __forceinline__ bool on_input(uint32_t) const { return true; }
    __device__ __forceinline__ Pre prepare(uint32_t, uint32_t, uint32_t v) const {
        return Pre{__ldcg(&level[v])};
    }
    // claims first (all issued before any result is used), then the outcomes
    template <int N>
    __device__ __forceinline__ void apply_n(const Pre (&p)[N], const uint32_t (&v)[N],
                                            int (&act)[N]) {
        int r[N];
#pragma unroll
        for (int j = 0; j < N; j++) {
            act[j] = act[j] && p[j].lvl == kInf;
            r[j] = act[j] ? atomicCAS(&level[v[j]], kInf, next) : 0;
        }
#pragma unroll
        for (int j = 0; j < N; j++) act[j] = act[j] && r[j] == kInf;
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
    c->ncand[0] = 0;   // pull candidate list
    c->ncand[1] = 0;   // pull overflow list
    if (c->mode == 0 && c->queue_stale) c->qsize[c->cur] = 0;   // rebuilt from the bitmap
}

// Pull lists, built once per graph by bfs_pull_lists.
struct PullLists {
    uint32_t V;
    const uint32_t *pidx;      // in-edges, highest out-degree source first
    const uint32_t *first;     // pidx[colptr[v]] (v's likeliest parent), or kNoParent
    const uint32_t *order;     // vertices by in-degree (heavy: in-degree > kPullHeavy)
    uint32_t n_heavy, n_light;
    uint32_t *cand;            // vertices whose first probe failed (V entries)
    uint32_t *ovf;             // candidates with in-edges left after the group pass
    uint32_t *fb0, *fb1;
    uint32_t words;            // words per bitmap
};

constexpr uint32_t kPullHeavy = 128;   // in-degree split of the sorted vertex list
constexpr uint32_t kNoParent = 0xffffffffu;
constexpr uint32_t kGroupProbe = 8;    // in-edges 1..8 probed by the candidate pass

// Four consecutive vertices per thread: v0 = 4 * quad.  Loads level[v0..v0+3]
// as one int4 when the array is 16-byte aligned and the quad is complete, else
// one int at a time; vertices >= V read as visited (0).
__device__ __forceinline__ int4 load_quad_level(const int32_t *level, uint64_t v0, uint32_t V,
                                                bool vec) {
    if (vec && v0 + 3 < V) return __ldcg(reinterpret_cast<const int4 *>(level + v0));
    int4 r = make_int4(0, 0, 0, 0);
    if (v0 < V) r.x = __ldcg(level + v0);
    if (v0 + 1 < V) r.y = __ldcg(level + v0 + 1);
    if (v0 + 2 < V) r.z = __ldcg(level + v0 + 2);
    if (v0 + 3 < V) r.w = __ldcg(level + v0 + 3);
    return r;
}

// The 32-bit bitmap word of the 8 quads held by lanes 8k..8k+7: each lane
// contributes its 4-bit nibble; lane 8k gets the whole word.
__device__ __forceinline__ uint32_t quad_word(uint32_t nibble) {
    uint32_t w = nibble << ((lane_id() & 7) * 4);
    w |= __shfl_xor_sync(0xffffffffu, w, 1);
    w |= __shfl_xor_sync(0xffffffffu, w, 2);
    w |= __shfl_xor_sync(0xffffffffu, w, 4);
    return w;
}

// Pull-level preparation, when the previous level was a push level: the
// current frontier's bitmap (level == L) from the level array, one whole word
// per 8 lanes.
__global__ void __launch_bounds__(kBlock)
k_bfs_pull_prep(uint32_t V, TravCtl *c, PullLists p) {
    if (c->done || c->mode != 1 || c->fb_valid) return;
    const int32_t *level = static_cast<const int32_t *>(c->vdata);
    const int L = (int)c->level;
    uint32_t *fcur = c->fb_cur ? p.fb1 : p.fb0;
    const bool vec = ((uintptr_t)level & 15) == 0;
    const uint64_t nw = ((uint64_t)V + 31) / 32, nquad = nw * 8;
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < nquad;
         base += (uint64_t)gridDim.x * kBlock) {
        const uint64_t qd = base + threadIdx.x;
        const int4 lv = load_quad_level(level, qd * 4, V, vec);
        const uint32_t nib = (lv.x == L) | (lv.y == L) << 1 | (lv.z == L) << 2 | (lv.w == L) << 3;
        const uint32_t w = quad_word(nib);
        if ((lane_id() & 7) == 0 && qd < nquad) fcur[qd >> 3] = w;
    }
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

// Pull, pass 1.  Each thread takes four consecutive vertices and does one
// probe per unvisited one: its first in-edge (first[v], the in-neighbour of
// highest out-degree, the one a BFS reaches earliest) against the frontier
// bitmap.  Every load is a coalesced vector load except the bitmap probe,
// which hits a 2 MB bitmap held in L2; the four vertices' loads are issued
// together.  A vertex whose first probe fails and that has more in-edges goes
// to the candidate list.  Lanes 8k..8k+7 own one 32-vertex word of the next
// bitmap and store it whole, so the next bitmap needs no clearing and no
// atomics in this pass.
__global__ void __launch_bounds__(kBlock)
k_bfs_pull(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowptr,
           TravCtl *c, PullLists p) {
    if (c->done || c->mode != 1) return;
    int32_t *level = static_cast<int32_t *>(c->vdata);
    const int L = (int)c->level;
    const uint32_t V = p.V;
    const uint32_t *__restrict__ fin = c->fb_cur ? p.fb1 : p.fb0;
    uint32_t *fout = c->fb_cur ? p.fb0 : p.fb1;
    const bool vec = ((uintptr_t)level & 15) == 0;
    const uint32_t wl = threadIdx.x >> 5;
    __shared__ uint32_t s_c[kBlock / 32][kWarpStage];
    __shared__ uint32_t s_cn[kBlock / 32], s_clim[kBlock / 32];
    if (lane_id() == 0) {
        s_cn[wl] = 0;
        s_clim[wl] = kWarpStage;
    }
    __syncwarp();
    unsigned long long acc = 0, nfound = 0;
    const uint64_t nw = ((uint64_t)V + 31) / 32, nquad = nw * 8;
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < nquad;
         base += (uint64_t)gridDim.x * kBlock) {
        const uint64_t qd = base + threadIdx.x;
        const uint64_t v0 = qd * 4;
        const int4 lv = load_quad_level(level, v0, V, vec);
        uint32_t um = (lv.x == kInf) | (lv.y == kInf) << 1 | (lv.z == kInf) << 2 |
                      (lv.w == kInf) << 3;
        uint32_t fm = 0, cm = 0;
        if (um) {
            uint4 f;
            if (v0 + 3 < V) {
                f = __ldg(reinterpret_cast<const uint4 *>(p.first + v0));
            } else {
                f = make_uint4(kNoParent, kNoParent, kNoParent, kNoParent);
                if (v0 < V) f.x = __ldg(p.first + v0);
                if (v0 + 1 < V) f.y = __ldg(p.first + v0 + 1);
                if (v0 + 2 < V) f.z = __ldg(p.first + v0 + 2);
            }
            const uint32_t fa[4] = {f.x, f.y, f.z, f.w};
            bool hit[4];
#pragma unroll
            for (int j = 0; j < 4; j++)
                hit[j] = ((um >> j) & 1) && fa[j] != kNoParent && in_bitmap(fin, fa[j]);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (hit[j]) fm |= 1u << j;
                else if (((um >> j) & 1) && fa[j] != kNoParent) cm |= 1u << j;
            }
        }
        if (fm) {
            // rowptr[v0..v0+4]: out-degrees of the new frontier vertices
            uint32_t r[5];
#pragma unroll
            for (int j = 0; j < 5; j++) r[j] = (fm >> j & 1) || (j > 0 && (fm >> (j - 1) & 1))
                                                   ? __ldg(&rowptr[v0 + j]) : 0;
            int4 out = lv;
            if (fm & 1) out.x = L + 1;
            if (fm & 2) out.y = L + 1;
            if (fm & 4) out.z = L + 1;
            if (fm & 8) out.w = L + 1;
            if (vec && v0 + 3 < V) {
                *reinterpret_cast<int4 *>(level + v0) = out;
            } else {
                if (fm & 1) level[v0] = L + 1;
                if (fm & 2) level[v0 + 1] = L + 1;
                if (fm & 4) level[v0 + 2] = L + 1;
                if (fm & 8) level[v0 + 3] = L + 1;
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (fm >> j & 1) acc += r[j + 1] - r[j];
            nfound += __popc(fm);
        }
        if (cm) {
            // candidates with one in-edge have no other parent to try
            uint32_t cp[5];
#pragma unroll
            for (int j = 0; j < 5; j++) cp[j] = (cm >> j & 1) || (j > 0 && (cm >> (j - 1) & 1))
                                                    ? __ldg(&colptr[v0 + j]) : 0;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if ((cm >> j & 1) && cp[j + 1] - cp[j] < 2) cm &= ~(1u << j);
        }
        const uint32_t w = quad_word(fm);
        if ((lane_id() & 7) == 0 && qd < nquad) fout[qd >> 3] = w;
        int act[4];
        uint32_t vv[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            act[j] = (cm >> j) & 1;
            vv[j] = (uint32_t)(v0 + j);
        }
        __syncwarp();
        if (s_cn[wl] + 32 * 4 > kWarpStage)
            warp_stage_flush(s_c[wl], &s_cn[wl], &s_clim[wl], p.cand, &c->ncand[0]);
        stage_push_n<4>(act, vv, 1, s_c[wl], &s_cn[wl], &s_clim[wl], kWarpStage, p.cand,
                        &c->ncand[0]);
    }
    warp_stage_flush(s_c[wl], &s_cn[wl], &s_clim[wl], p.cand, &c->ncand[0]);
    warp_add64(acc, &c->m_next);
    // the next frontier lives in the bitmap; only its size is counted here
    warp_add64(nfound, &c->reached_pull);
}

// Pull, pass 2: eight lanes per candidate probe in-edges 1..8 at once (one
// 32-byte sector of the in-edge list).  A candidate with in-edges left after
// that goes to the overflow list.
__global__ void __launch_bounds__(kBlock)
k_bfs_pull_cand(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowptr,
                TravCtl *c, PullLists p) {
    if (c->done || c->mode != 1) return;
    const uint32_t n = c->ncand[0];
    if (n == 0) return;
    int32_t *level = static_cast<int32_t *>(c->vdata);
    const int L = (int)c->level;
    const uint32_t *__restrict__ fin = c->fb_cur ? p.fb1 : p.fb0;
    uint32_t *fout = c->fb_cur ? p.fb0 : p.fb1;
    const uint32_t lane = lane_id(), sub = lane & 7, grp = lane & 24;
    const uint32_t gwarp = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kBlock) >> 5;
    unsigned long long acc = 0, nfound = 0;
    for (uint64_t base = (uint64_t)gwarp * 4; base < n; base += (uint64_t)nwarps * 4) {
        const uint64_t i = base + (lane >> 3);
        const bool valid = i < n;
        uint32_t v = 0, b = 0, e = 0;
        if (valid) {
            v = p.cand[i];
            b = __ldg(&colptr[v]) + 1;
            e = __ldg(&colptr[v + 1]);
        }
        const uint32_t j = b + sub;
        const bool hit = valid && j < e && in_bitmap(fin, __ldg(&p.pidx[j]));
        const uint32_t gm = (__ballot_sync(0xffffffffu, hit) >> grp) & 0xffu;
        const bool more = valid && !gm && e > b + kGroupProbe;
        if (valid && gm && sub == 0) {
            level[v] = L + 1;
            atomicOr(&fout[v >> 5], 1u << (v & 31));
            acc += __ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]);
            nfound++;
        }
        warp_push(more && sub == 0, v, p.ovf, &c->ncand[1]);
    }
    warp_add64(acc, &c->m_next);
    warp_add64(nfound, &c->reached_pull);
}

// Pull, pass 3: one warp per overflow vertex scans the rest of its in-edges,
// 32 per probe, and stops at the first parent.
__global__ void __launch_bounds__(kBlock)
k_bfs_pull_overflow(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowptr,
                    TravCtl *c, PullLists p) {
    if (c->done || c->mode != 1) return;
    const uint32_t n = c->ncand[1];
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
        const uint32_t v = p.ovf[i];
        const uint32_t b = __ldg(&colptr[v]) + 1 + kGroupProbe, e = __ldg(&colptr[v + 1]);
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
        // hub pieces of one superstep: at most E/piece + (rows over hub_degree),
        // for the BFS and the SSSP settings alike
        const Tuning &t = g->tune;
        const uint64_t piece = t.piece < t.sssp_piece ? t.piece : t.sssp_piece;
        const uint64_t hub = t.hub_degree < t.sssp_hub_degree ? t.hub_degree : t.sssp_hub_degree;
        const uint64_t np = g->E / piece + g->E / hub + 16;
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

// first[v] = v's first in-edge in pull order (its highest out-degree
// in-neighbour), kNoParent for a vertex without in-edges.
__global__ void k_first_parent(const uint32_t *__restrict__ colptr,
                               const uint32_t *__restrict__ pidx, uint32_t V,
                               uint32_t *__restrict__ first) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = colptr[v], e = colptr[v + 1];
        first[v] = b < e ? pidx[b] : kNoParent;
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
    OLV_TRY(w.cand.ensure((size_t)V * 4 + 16));    // pull candidate list
    OLV_TRY(w.cand2.ensure((size_t)V * 4 + 16));   // pull overflow list
    OLV_TRY(w.pull_first.ensure((size_t)V * 4 + 16));
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
    }
    k_first_parent<<<g->num_sms * 8, kBlock, 0, s>>>(g->colptr.as<uint32_t>(),
                                                    w.pull_idx.as<uint32_t>(), V,
                                                    w.pull_first.as<uint32_t>());
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaStreamSynchronize(s));
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
    pl.first = g->ws.pull_first.as<uint32_t>();
    pl.cand = g->ws.cand.as<uint32_t>();
    pl.ovf = g->ws.cand2.as<uint32_t>();
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
    void *a_pull[] = {&colptr, &rowptr, &ctl, &pl};
    OLV_TRY(sink((const void *)k_bfs_pull, dim3(nb), dim3(kBlock), a_pull));
    OLV_TRY(sink((const void *)k_bfs_pull_cand, dim3(nb), dim3(kBlock), a_pull));
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
