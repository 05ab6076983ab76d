// Batched traversal of many small graphs packed block-diagonally in one CSR,
// run by ONE persistent kernel with a device-side work queue (no reference
// counterpart; each instance's result equals its solo run, bit for bit).
//
// Work items are (instance, task) pairs handed out by an atomic counter,
// largest instances first.  A CTA runs its item to completion:
//   BFS from the instance's local vertex 0 (testBFS.cu semantics, levels
//     relative to the instance, 0x7fffffff unreached).  The visited, current
//     and next frontier bitmaps of the instance live in shared memory
//     (3 x 8 KB for up to 65,536 vertices); a thread per vertex expands the
//     frontier with shared-memory atomicOr claims.
//   PPR: K <= 32 personalised PageRank vectors with one-hot seeds (the
//     oracle's orc_ppr definition: dangling mass returns to the seed), pulled
//     over the in-edges with one warp per vertex and lane k = vector k, so
//     each in-edge reads one 128-byte row, scaled by the source's inverse
//     out-degree (computed once per item).  A warp keeps eight rows in
//     flight; sums still run in CSC order per lane, the dangling mass is
//     summed while the new vectors are written, and cross-warp reductions
//     run in a fixed order, so results do not depend on which CTA runs the
//     item or when.  Stops after max_it iterations or when every vector's L1
//     change (FP64) is below tol.
#include <algorithm>
#include <numeric>
#include <vector>

#include <cooperative_groups.h>

#include "olive_b200/olv_advance.cuh"
#include "olv_internal.cuh"

namespace cg = cooperative_groups;

namespace olv {

constexpr int kBatchThreads = 512;
constexpr uint32_t kBatchMaxV = 65536;
constexpr int kBatchWarps = kBatchThreads / 32;

struct BatchArgs {
    const uint32_t *rowptr, *col, *colptr, *rowidx;
    const uint32_t *inst_off;
    const uint32_t *order;       // instances, largest first
    const uint32_t *seeds;       // [count][K] local ids
    int count, K, max_it, tasks; // tasks: 1 = BFS only / PPR only, 2 = both
    int do_bfs, do_ppr;
    float alpha;
    double tol;
    int32_t *levels;             // [V]
    float *ppr, *ppr_tmp;        // [V][K]
    float *inv_deg;              // [V] 1 / out-degree (0: dangling), written per PPR item
    uint32_t *counter;           // work queue head
    uint32_t *ppr_iters;         // [count]
    unsigned long long *stats;   // [0] BFS edges traversed, [1] PPR edge visits, [2] error bits
};

__device__ void cta_bfs(const BatchArgs &a, uint32_t inst, uint32_t *bm) {
    const uint32_t base = a.inst_off[inst], n = a.inst_off[inst + 1] - base;
    const uint32_t words = (n + 31) / 32;
    uint32_t *vis = bm, *cur = bm + kBatchMaxV / 32, *nxt = bm + 2 * (kBatchMaxV / 32);
    __shared__ int s_any;
    __shared__ unsigned long long s_edges;
    for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) {
        vis[w] = 0;
        cur[w] = 0;
    }
    for (uint32_t v = threadIdx.x; v < n; v += blockDim.x) a.levels[base + v] = kInf;
    __syncthreads();
    if (threadIdx.x == 0) {
        vis[0] = 1u;
        cur[0] = 1u;
        a.levels[base] = 0;
        s_edges = 0;
    }
    unsigned long long edges = 0;
    for (int L = 0;; L++) {
        for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) nxt[w] = 0;
        if (threadIdx.x == 0) s_any = 0;
        __syncthreads();
        int any = 0;
        for (uint32_t u = threadIdx.x; u < n; u += blockDim.x) {
            if (!((cur[u >> 5] >> (u & 31)) & 1u)) continue;
            const uint32_t b = a.rowptr[base + u], e = a.rowptr[base + u + 1];
            edges += e - b;
            for (uint32_t i = b; i < e; i++) {
                const uint32_t v = a.col[i] - base;
                if (v >= n) {   // edge leaves the instance: not block-diagonal
                    atomicOr((unsigned int *)&a.stats[2], 1u);
                    continue;
                }
                const uint32_t bit = 1u << (v & 31);
                if (vis[v >> 5] & bit) continue;
                if (!(atomicOr(&vis[v >> 5], bit) & bit)) {
                    atomicOr(&nxt[v >> 5], bit);
                    a.levels[base + v] = L + 1;
                    any = 1;
                }
            }
        }
        if (any) s_any = 1;
        __syncthreads();
        uint32_t *t = cur;
        cur = nxt;
        nxt = t;
        const int go = s_any;
        __syncthreads();
        if (!go) break;
    }
    atomicAdd(&s_edges, edges);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&a.stats[0], s_edges);
    __syncthreads();
}

// Rows gathered per round of one warp's in-edge walk: the loads of a round
// are issued together, then folded in CSC order.
constexpr int kPprRound = 8;

// What one warp sees of a PPR item.
struct PprView {
    uint32_t base, n, seed;
    int K;
    bool lk;          // lane < K: the lane carries vector `lane`
    float alpha;
    float *r0, *r1;   // the item's vectors, ping-pong
    float *inv;       // 1 / out-degree, 0 for a dangling vertex
};

__device__ __forceinline__ PprView ppr_view(const BatchArgs &a, uint32_t inst, uint32_t lane) {
    PprView p;
    p.base = a.inst_off[inst];
    p.n = a.inst_off[inst + 1] - p.base;
    p.K = a.K;
    p.lk = (int)lane < p.K;
    p.seed = p.lk ? a.seeds[(size_t)inst * p.K + lane] : 0xffffffffu;
    p.alpha = a.alpha;
    p.r0 = a.ppr + (size_t)p.base * p.K;
    p.r1 = a.ppr_tmp + (size_t)p.base * p.K;
    p.inv = a.inv_deg + p.base;
    return p;
}

// Start vectors and inverse out-degrees of the vertices v = w0, w0 + nw, ...;
// returns this warp's dangling mass of the start vectors (per lane), summed
// in vertex order.
__device__ __forceinline__ float ppr_init_warp(const BatchArgs &a, const PprView &p, uint32_t lane,
                                               uint32_t w0, uint32_t nw) {
    float dpart = 0.0f;
    for (uint32_t v = w0; v < p.n; v += nw) {
        const uint32_t deg = a.rowptr[p.base + v + 1] - a.rowptr[p.base + v];
        if (lane == 0) p.inv[v] = deg ? __fdiv_rn(1.0f, (float)deg) : 0.0f;
        const float x = (v == p.seed) ? 1.0f : 0.0f;
        if (p.lk) p.r0[(size_t)v * p.K + lane] = x;
        if (!deg) dpart += x;
    }
    return dpart;
}

// One sweep over the vertices v = w0, w0 + nw, ... (one warp each): pull
// src over the in-edges, write dst; accumulates the warp's dangling mass of
// the new vectors, its FP64 L1 change and its in-edge visits.
__device__ __forceinline__ void ppr_sweep_warp(const BatchArgs &a, const PprView &p, uint32_t lane,
                                               uint32_t w0, uint32_t nw, const float *src,
                                               float *dst, float dk, float &dpart, double &res,
                                               unsigned long long &visits) {
    const uint32_t base = p.base, n = p.n;
    const int K = p.K;
    for (uint32_t v = w0; v < n; v += nw) {
        const uint32_t b = a.colptr[base + v], e = a.colptr[base + v + 1];
        float acc = 0.0f;
        // 32 in-edges at a time: lane j fetches source j and its inverse
        // degree, then the warp gathers the sources' rows kPprRound at a
        // time (lane k = vector k) and folds them in CSC order.  Padding
        // slots carry weight 0 and add exactly 0.
        for (uint32_t c0 = b; c0 < e; c0 += 32) {
            const uint32_t cnt = min(32u, e - c0);
            uint32_t u = 0;
            float w = 0.0f;
            if (lane < cnt) {
                u = a.rowidx[c0 + lane] - base;
                if (u >= n) {   // edge enters from outside the instance
                    atomicOr((unsigned int *)&a.stats[2], 2u);
                    u = 0;
                } else {
                    w = p.inv[u];
                }
            }
            for (uint32_t t = 0; t < cnt; t += kPprRound) {
                float x[kPprRound], ww[kPprRound];
#pragma unroll
                for (int j = 0; j < kPprRound; j++) {
                    const uint32_t uj = __shfl_sync(0xffffffffu, u, (t + j) & 31);
                    ww[j] = __shfl_sync(0xffffffffu, w, (t + j) & 31);
                    x[j] = (p.lk && t + j < cnt) ? src[(size_t)uj * K + lane] : 0.0f;
                }
#pragma unroll
                for (int j = 0; j < kPprRound; j++)
                    if (t + j < cnt) acc = fmaf(x[j], ww[j], acc);
            }
        }
        visits += e - b;
        if (p.lk) {
            const float tele = (v == p.seed) ? fmaf(p.alpha, dk, 1.0f - p.alpha) : 0.0f;
            const float nv = fmaf(p.alpha, acc, tele);
            res += fabs((double)nv - (double)src[(size_t)v * K + lane]);
            dst[(size_t)v * K + lane] = nv;
            if (p.inv[v] == 0.0f) dpart += nv;
        }
    }
}

#ifndef OLV_QROUND
#define OLV_QROUND 4
#endif
constexpr int kQRound = OLV_QROUND;   // in-edges per vertex gathered per round

// K = 32 sweep with four vertices per warp: slot s = lane >> 3 (8 lanes)
// takes vertex 4g + s of vertex group g (g = w0, w0 + nw, ...), lane quad q =
// lane & 7 holds vectors 4q .. 4q+3 of it as one float4.  A round gathers
// two in-edges of each of the four vertices (one 16-byte load per lane per
// in-edge), so the per-vertex work -- offsets, sources, update, residual --
// is shared by four vertices per instruction.  Each vertex's in-edges are
// folded in CSC order; the warp's dangling mass and L1 change are combined
// over the slots by a fixed shuffle tree and returned in the lane-per-vector
// layout, like ppr_sweep_warp.  `visits` gets the warp's in-edge visits.
// Needs 16-byte aligned vectors.  Used by the cluster kernel, whose rows come
// from L2 (the one-CTA-per-item kernel is bound by DRAM traffic and keeps the
// 4-byte path).
__device__ __forceinline__ void ppr_sweep_warp_q(const BatchArgs &a, const PprView &p,
                                                 uint32_t lane, uint32_t w0, uint32_t nw,
                                                 const float *src, float *dst, float dk,
                                                 float &dpart, double &res,
                                                 unsigned long long &visits) {
    constexpr unsigned kFull = 0xffffffffu;
    const uint32_t base = p.base, n = p.n;
    const uint32_t slot = lane >> 3, quad = lane & 7;
    const float4 *src4 = reinterpret_cast<const float4 *>(src);
    float4 *dst4 = reinterpret_cast<float4 *>(dst);
    uint32_t seed4[4];
    float dk4[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        seed4[c] = __shfl_sync(kFull, p.seed, 4 * quad + c);
        dk4[c] = __shfl_sync(kFull, dk, 4 * quad + c);
    }
    float dp4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    double rs4[4] = {0.0, 0.0, 0.0, 0.0};
    unsigned long long vq = 0;
    for (uint32_t g = w0; 4 * g < n; g += nw) {
        const uint32_t v = 4 * g + slot;
        const bool valid = v < n;
        uint32_t b = 0, deg = 0;
        if (valid) {
            b = a.colptr[base + v];
            deg = a.colptr[base + v + 1] - b;
        }
        uint32_t maxdeg = deg;
        maxdeg = max(maxdeg, __shfl_xor_sync(kFull, maxdeg, 8));
        maxdeg = max(maxdeg, __shfl_xor_sync(kFull, maxdeg, 16));
        float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (uint32_t c0 = 0; c0 < maxdeg; c0 += 8) {
            // lane quad q of a slot holds in-edge c0 + q of the slot's vertex
            uint32_t u = 0;
            float w = 0.0f;
            if (c0 + quad < deg) {
                u = a.rowidx[b + c0 + quad] - base;
                if (u >= n) {   // edge enters from outside the instance
                    atomicOr((unsigned int *)&a.stats[2], 2u);
                    u = 0;
                } else {
                    w = p.inv[u];
                }
            }
            const uint32_t cend = min(8u, maxdeg - c0);
            for (uint32_t t = 0; t < cend; t += kQRound) {
                float4 x[kQRound];
                float wj[kQRound];
#pragma unroll
                for (int r = 0; r < kQRound; r++) {
                    const uint32_t i = t + r;
                    const uint32_t uj = __shfl_sync(kFull, u, slot * 8 + (i & 7));
                    wj[r] = __shfl_sync(kFull, w, slot * 8 + (i & 7));
                    x[r] = c0 + i < deg ? src4[(size_t)uj * 8 + quad]
                                        : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                }
#pragma unroll
                for (int r = 0; r < kQRound; r++) {
                    if (c0 + t + r < deg) {
                        acc.x = fmaf(x[r].x, wj[r], acc.x);
                        acc.y = fmaf(x[r].y, wj[r], acc.y);
                        acc.z = fmaf(x[r].z, wj[r], acc.z);
                        acc.w = fmaf(x[r].w, wj[r], acc.w);
                    }
                }
            }
        }
        if (quad == 0) vq += deg;
        if (valid) {
            const float4 old = src4[(size_t)v * 8 + quad];
            const float a4[4] = {acc.x, acc.y, acc.z, acc.w};
            const float o4[4] = {old.x, old.y, old.z, old.w};
            float nv[4];
            const bool dang = p.inv[v] == 0.0f;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float tele = (v == seed4[c]) ? fmaf(p.alpha, dk4[c], 1.0f - p.alpha) : 0.0f;
                nv[c] = fmaf(p.alpha, a4[c], tele);
                rs4[c] += fabs((double)nv[c] - (double)o4[c]);
                if (dang) dp4[c] += nv[c];
            }
            dst4[(size_t)v * 8 + quad] = make_float4(nv[0], nv[1], nv[2], nv[3]);
        }
    }
    // slots 0+1 and 2+3, then the pairs; back to lane k = vector k
#pragma unroll
    for (int o = 8; o <= 16; o <<= 1) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            dp4[c] += __shfl_xor_sync(kFull, dp4[c], o);
            rs4[c] += __shfl_xor_sync(kFull, rs4[c], o);
        }
        vq += __shfl_xor_sync(kFull, vq, o);
    }
    const uint32_t from = lane >> 2, comp = lane & 3;
    float dsel = 0.0f;
    double rsel = 0.0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float dc = __shfl_sync(kFull, dp4[c], from);
        const double rc = __shfl_sync(kFull, rs4[c], from);
        if (comp == (uint32_t)c) {
            dsel = dc;
            rsel = rc;
        }
    }
    dpart += dsel;
    res += rsel;
    visits += vq;
}

// Whether an item's sweeps can use the 16-byte row path.
__device__ __forceinline__ bool ppr_v4(const BatchArgs &a) {
    return a.K == 32 && ((reinterpret_cast<uintptr_t>(a.ppr) | reinterpret_cast<uintptr_t>(a.ppr_tmp)) & 15) == 0;
}

__device__ void cta_ppr(const BatchArgs &a, uint32_t inst) {
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const PprView p = ppr_view(a, inst, lane);
    const uint32_t n = p.n;
    const int K = p.K;
    __shared__ float s_d[kBatchWarps][32];
    __shared__ double s_res[kBatchWarps][32];
    __shared__ float s_dang[32];
    __shared__ int s_stop;
    // Dangling mass is always summed in the same order: each warp over its
    // vertices (v = wid, wid + W, ...), then warps 0..W-1.
    s_d[wid][lane] = ppr_init_warp(a, p, lane, wid, kBatchWarps);
    __syncthreads();
    int it = 0;
    unsigned long long visits = 0;
    while (it < a.max_it) {
        const float *src = (it & 1) ? p.r1 : p.r0;
        float *dst = (it & 1) ? p.r0 : p.r1;
        if (wid == 0) {
            float t = 0.0f;
            for (int w = 0; w < kBatchWarps; w++) t += s_d[w][lane];
            s_dang[lane] = t;
        }
        __syncthreads();
        const float dk = s_dang[lane];
        double res = 0.0;
        float dpart = 0.0f;
        ppr_sweep_warp(a, p, lane, wid, kBatchWarps, src, dst, dk, dpart, res, visits);
        s_d[wid][lane] = dpart;
        s_res[wid][lane] = res;
        __syncthreads();
        if (threadIdx.x == 0) {
            double mx = 0.0;
            for (int k = 0; k < K; k++) {
                double t = 0.0;
                for (int w = 0; w < kBatchWarps; w++) t += s_res[w][k];
                mx = t > mx ? t : mx;
            }
            s_stop = mx < a.tol;
        }
        __syncthreads();
        it++;
        if (s_stop) break;
    }
    if (it & 1) {   // result is in the scratch copy
        for (uint32_t v = wid; v < n; v += kBatchWarps)
            if (p.lk) p.r0[(size_t)v * K + lane] = p.r1[(size_t)v * K + lane];
    }
    if (threadIdx.x == 0) a.ppr_iters[inst] = it;
    if (lane == 0 && visits) atomicAdd(&a.stats[1], visits * (unsigned long long)K);
    __syncthreads();
}

__global__ void __launch_bounds__(kBatchThreads) k_batch(BatchArgs a) {
    __shared__ uint32_t bm[3 * (kBatchMaxV / 32)];
    __shared__ uint32_t s_item;
    const uint32_t n_items = (uint32_t)a.count * a.tasks;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        __syncthreads();
        if (item >= n_items) break;
        const uint32_t inst = a.order[item / a.tasks];
        const bool bfs = a.tasks == 2 ? (item % 2 == 0) : (a.do_bfs != 0);
        if (bfs)
            cta_bfs(a, inst, bm);
        else
            cta_ppr(a, inst);
    }
}

// ---- cluster version ------------------------------------------------------
// The same items, with every PPR item run by a whole thread-block cluster
// (16 CTAs of 1024 threads where the GPU allows it, else 8): the cluster's
// 512 (256) warps split the instance's vertices, and the per-iteration
// reductions go through distributed shared memory with one cluster barrier
// per iteration.  Only a handful of instances are in flight at a time, so
// their PPR vectors (2 x V_i x 128 B each) stay in L2 and the 128-byte row
// gathers, eight per vertex per iteration, hit L2 instead of DRAM.  BFS items
// still take one CTA each, before the PPR items.  Results depend on the
// cluster size (it fixes the order of the dangling-mass sums), never on
// scheduling: a solo run with the same cluster size is bitwise equal.
constexpr int kClusterThreads = 1024;
constexpr int kClusterWarps = kClusterThreads / 32;

struct ClusterShared {
    float d[kClusterWarps][32];      // per-warp dangling mass
    double res[kClusterWarps][32];   // per-warp L1 change
    float dc[2][32];                 // CTA dangling mass, by iteration parity
    double rc[2][32];                // CTA L1 change, by iteration parity
    int stop;
};

__device__ void cluster_ppr(const BatchArgs &a, uint32_t inst, cg::cluster_group &cl,
                            ClusterShared &sh) {
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t C = cl.num_blocks(), crank = cl.block_rank();
    const uint32_t gw = crank * kClusterWarps + wid, nw = C * kClusterWarps;
    const PprView p = ppr_view(a, inst, lane);
    const int K = p.K;
    // dangling mass: each warp in vertex order, then warps 0..31 of a CTA,
    // then CTAs 0..C-1 (every CTA forms the same sum)
    sh.d[wid][lane] = ppr_init_warp(a, p, lane, gw, nw);
    __syncthreads();
    if (wid == 0) {
        float t = 0.0f;
        for (int w = 0; w < kClusterWarps; w++) t += sh.d[w][lane];
        sh.dc[0][lane] = t;
    }
    cl.sync();
    int it = 0;
    unsigned long long visits = 0;
    while (it < a.max_it) {
        const int pb = it & 1;
        float dk = 0.0f;
        for (uint32_t r = 0; r < C; r++) dk += cl.map_shared_rank(&sh.dc[pb][0], r)[lane];
        const float *src = pb ? p.r1 : p.r0;
        float *dst = pb ? p.r0 : p.r1;
        double res = 0.0;
        float dpart = 0.0f;
        if (ppr_v4(a))
            ppr_sweep_warp_q(a, p, lane, gw, nw, src, dst, dk, dpart, res, visits);
        else
            ppr_sweep_warp(a, p, lane, gw, nw, src, dst, dk, dpart, res, visits);
        sh.d[wid][lane] = dpart;
        sh.res[wid][lane] = res;
        __syncthreads();
        if (wid == 0) {
            float t = 0.0f;
            double q = 0.0;
            for (int w = 0; w < kClusterWarps; w++) {
                t += sh.d[w][lane];
                q += sh.res[w][lane];
            }
            sh.dc[pb ^ 1][lane] = t;
            sh.rc[pb ^ 1][lane] = q;
        }
        // orders this sweep's writes (vectors and partials) before every
        // CTA's reads of the next sweep, cluster wide
        cl.sync();
        if (wid == 0) {   // stop test: the same on every CTA
            double tot = 0.0;
            for (uint32_t r = 0; r < C; r++) tot += cl.map_shared_rank(&sh.rc[pb ^ 1][0], r)[lane];
            double mx = (int)lane < K ? tot : 0.0;
#pragma unroll
            for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0) sh.stop = mx < a.tol;
        }
        __syncthreads();
        it++;
        if (sh.stop) break;
    }
    if (it & 1) {   // result is in the scratch copy
        for (uint32_t v = gw; v < p.n; v += nw)
            if (p.lk) p.r0[(size_t)v * K + lane] = p.r1[(size_t)v * K + lane];
    }
    if (crank == 0 && threadIdx.x == 0) a.ppr_iters[inst] = it;
    if (lane == 0 && visits) atomicAdd(&a.stats[1], visits * (unsigned long long)K);
}

__global__ void __launch_bounds__(kClusterThreads, 1) k_batch_cluster(BatchArgs a) {
    __shared__ uint32_t bm[3 * (kBatchMaxV / 32)];
    __shared__ ClusterShared sh;
    __shared__ uint32_t s_item;
    cg::cluster_group cl = cg::this_cluster();
    if (a.do_bfs) {   // BFS items: one CTA each (counter[0])
        for (;;) {
            if (threadIdx.x == 0) s_item = atomicAdd(&a.counter[0], 1u);
            __syncthreads();
            const uint32_t item = s_item;
            __syncthreads();
            if (item >= (uint32_t)a.count) break;
            cta_bfs(a, a.order[item], bm);
        }
    }
    if (a.do_ppr) {   // PPR items: one cluster each (counter[1], taken by CTA 0)
        for (;;) {
            if (cl.block_rank() == 0 && threadIdx.x == 0) s_item = atomicAdd(&a.counter[1], 1u);
            cl.sync();
            const uint32_t item = *cl.map_shared_rank(&s_item, 0);
            if (item >= (uint32_t)a.count) break;
            cluster_ppr(a, a.order[item], cl, sh);
        }
    }
    cl.sync();   // no CTA leaves while another may still read its shared memory
}

// Launch k_batch_cluster with `want` CTAs per cluster (8 or 16), or with the
// largest size the GPU runs when want = 1; one CTA per SM.  *launched =
// false when no wanted size is available.
static int launch_batch_cluster(const BatchArgs &a, int num_sms, cudaStream_t s, int want,
                                bool *launched, int *cluster_size) {
    *launched = false;
    if (cudaFuncSetAttribute(k_batch_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
        cudaSuccess)
        cudaGetLastError();
    for (int C : {16, 8}) {
        if (want != 1 && want != C) continue;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(C * std::max(1, num_sms / C));
        cfg.blockDim = dim3(kClusterThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, k_batch_cluster, &cfg) != cudaSuccess || ncl < 1) {
            cudaGetLastError();
            continue;
        }
        cfg.gridDim = dim3(C * std::min(ncl, std::max(1, num_sms / C)));
        OLV_CUDA(cudaLaunchKernelEx(&cfg, k_batch_cluster, a));
        *launched = true;
        *cluster_size = C;
        return OLV_OK;
    }
    return OLV_OK;
}

// Device buffers of olv_batch_run, kept with the graph between calls (they
// only grow), so a call allocates nothing once the sizes have been seen.
struct BatchState {
    DevBuf off, order, seeds, tmp, inv, counter, iters, stats, levels, ppr;
    ~BatchState() {
        off.release(); order.release(); seeds.release(); tmp.release(); inv.release(); counter.release();
        iters.release(); stats.release(); levels.release(); ppr.release();
    }
};

void release_batch_state(olv_graph *g) {
    delete static_cast<BatchState *>(g->batch_state);
    g->batch_state = nullptr;
}

}  // namespace olv

using namespace olv;

extern "C" int olv_batch_run(olv_graph *g, const uint32_t *inst_offsets, int count, int K,
                             const uint32_t *seeds, double alpha, int max_it, double tol,
                             int32_t *levels_out, float *ppr_out, uint32_t *ppr_iters_out,
                             olv_stats *st) {
    OLV_CHECK_ARG(g && inst_offsets, "olv_batch_run: null pointer");
    OLV_CHECK_ARG(count >= 1, "olv_batch_run: count must be >= 1");
    OLV_CHECK_ARG(levels_out || ppr_out, "olv_batch_run: nothing to compute");
    OLV_CHECK_ARG(!ppr_out || (seeds && K >= 1 && K <= 32),
                  "olv_batch_run: PPR needs seeds and 1 <= K <= 32");
    OLV_CHECK_ARG(alpha >= 0 && alpha < 1 && max_it >= 0, "olv_batch_run: bad alpha / max_it");
    std::vector<uint32_t> off(count + 1);
    if (is_device_ptr(inst_offsets))
        OLV_CUDA(cudaMemcpy(off.data(), inst_offsets, (count + 1) * 4, cudaMemcpyDeviceToHost));
    else
        memcpy(off.data(), inst_offsets, (count + 1) * 4);
    OLV_CHECK_ARG(off[count] <= g->V, "olv_batch_run: offsets exceed the graph");
    for (int i = 0; i < count; i++) {
        OLV_CHECK_ARG(off[i + 1] > off[i], "olv_batch_run: empty or decreasing instance %d", i);
        if (off[i + 1] - off[i] > kBatchMaxV) {
            set_error("olv_batch_run: instance %d has %u vertices (limit %u)", i,
                      off[i + 1] - off[i], kBatchMaxV);
            return OLV_ERR_LIMIT;
        }
    }
    const int K_ = ppr_out ? K : 0;
    std::vector<uint32_t> hseeds;
    if (ppr_out) {
        hseeds.resize((size_t)count * K);
        if (is_device_ptr(seeds))
            OLV_CUDA(cudaMemcpy(hseeds.data(), seeds, hseeds.size() * 4, cudaMemcpyDeviceToHost));
        else
            memcpy(hseeds.data(), seeds, hseeds.size() * 4);
        for (int i = 0; i < count; i++)
            for (int k = 0; k < K; k++)
                OLV_CHECK_ARG(hseeds[(size_t)i * K + k] < off[i + 1] - off[i],
                              "olv_batch_run: seed %d of instance %d out of range", k, i);
    }
    // largest instances first
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        return off[x + 1] - off[x] > off[y + 1] - off[y];
    });
    if (!g->batch_state) g->batch_state = new BatchState();
    BatchState &bs = *static_cast<BatchState *>(g->batch_state);
    cudaStream_t s = g->stream;
    const size_t V = off[count];
    OLV_TRY(bs.off.ensure((count + 1) * 4));
    OLV_TRY(bs.order.ensure(count * 4));
    OLV_TRY(bs.counter.ensure(16));
    OLV_TRY(bs.iters.ensure(count * 4 + 16));
    OLV_TRY(bs.stats.ensure(32));
    OLV_CUDA(cudaMemcpyAsync(bs.off.p, off.data(), (count + 1) * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(bs.order.p, order.data(), count * 4, cudaMemcpyHostToDevice, s));
    const bool dev_lv = levels_out && is_device_ptr(levels_out);
    const bool dev_pr = ppr_out && is_device_ptr(ppr_out);
    if (levels_out && !dev_lv) OLV_TRY(bs.levels.ensure(V * 4));
    if (ppr_out) {
        OLV_TRY(bs.seeds.ensure(hseeds.size() * 4));
        OLV_CUDA(cudaMemcpyAsync(bs.seeds.p, hseeds.data(), hseeds.size() * 4,
                                 cudaMemcpyHostToDevice, s));
        OLV_TRY(bs.tmp.ensure(V * K * 4));
        OLV_TRY(bs.inv.ensure(V * 4));
        if (!dev_pr) OLV_TRY(bs.ppr.ensure(V * K * 4));
    }
    BatchArgs a;
    a.rowptr = g->rowptr.as<uint32_t>();
    a.col = g->col.as<uint32_t>();
    a.colptr = g->colptr.as<uint32_t>();
    a.rowidx = g->rowidx.as<uint32_t>();
    a.inst_off = bs.off.as<uint32_t>();
    a.order = bs.order.as<uint32_t>();
    a.seeds = bs.seeds.as<uint32_t>();
    a.count = count;
    a.K = K_;
    a.max_it = max_it;
    a.do_bfs = levels_out != nullptr;
    a.do_ppr = ppr_out != nullptr;
    a.tasks = a.do_bfs + a.do_ppr;
    a.alpha = (float)alpha;
    a.tol = tol;
    a.levels = levels_out ? (dev_lv ? levels_out : bs.levels.as<int32_t>()) : nullptr;
    a.ppr = ppr_out ? (dev_pr ? ppr_out : bs.ppr.as<float>()) : nullptr;
    a.ppr_tmp = bs.tmp.as<float>();
    a.inv_deg = bs.inv.as<float>();
    a.counter = bs.counter.as<uint32_t>();
    a.ppr_iters = bs.iters.as<uint32_t>();
    a.stats = bs.stats.as<unsigned long long>();
    OLV_CUDA(cudaEventRecord(g->ev0, s));
    OLV_CUDA(cudaMemsetAsync(bs.counter.p, 0, 16, s));
    OLV_CUDA(cudaMemsetAsync(bs.stats.p, 0, 32, s));
    bool launched = false;
    int csize = 0;
    if (g->tune.batch_cluster)
        OLV_TRY(launch_batch_cluster(a, g->num_sms, s, g->tune.batch_cluster, &launched, &csize));
    if (!launched) {   // one CTA per item
        int per_sm = 0;
        OLV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, kBatchThreads, 0));
        const int grid = std::max(1, per_sm) * g->num_sms;
        k_batch<<<grid, kBatchThreads, 0, s>>>(a);
    }
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    unsigned long long hst[3];
    OLV_CUDA(cudaMemcpyAsync(hst, bs.stats.p, 24, cudaMemcpyDeviceToHost, s));
    if (levels_out && !dev_lv)
        OLV_CUDA(cudaMemcpyAsync(levels_out, a.levels, V * 4, cudaMemcpyDeviceToHost, s));
    if (ppr_out && !dev_pr)
        OLV_CUDA(cudaMemcpyAsync(ppr_out, a.ppr, V * K * 4, cudaMemcpyDeviceToHost, s));
    if (ppr_iters_out)
        OLV_CUDA(cudaMemcpyAsync(ppr_iters_out, bs.iters.p, count * 4, cudaMemcpyDefault, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    if (hst[2]) {
        set_error("olv_batch_run: the graph is not block-diagonal under inst_offsets "
                  "(edges cross instances; code %llu)", hst[2]);
        return OLV_ERR_ARG;
    }
    if (st) {
        float ms = 0;
        OLV_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        st->iterations = (uint32_t)count;
        st->pull_steps = 0;
        st->vertices_reached = V;
        st->edges_traversed = hst[0];   // BFS: out-edges of reached vertices, all instances
        st->edges_relaxed = hst[1];     // PPR: in-edge visits x K, all iterations
        st->residual = 0;
        st->device_ms = ms;
    }
    return OLV_OK;
}
