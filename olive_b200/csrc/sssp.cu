// Single-source shortest paths with non-negative uint32 weights.
//
// Result contract: the frontier Bellman-Ford of SSSP.cu:106-174 run to
// convergence -- gather = dist[u] + w (SSSP.cu:54-57), reduce = atomicMin
// (SSSP.cu:60-63), a vertex re-enters the frontier when its distance drops
// (cond/update, SSSP.cu:66-76).  Distances are unique, so the result equals
// serial Dijkstra bit for bit; 0x7fffffff marks unreached vertices.
//
// B200 formulation: the same atomicMin relaxation, ordered as delta-stepping
// with a near queue and a far pile, and light/heavy edges (Meyer & Sanders):
//   * each row is stored light edges first (w <= delta), then heavy ones
//     (built once per graph and delta, k_partition_rows);
//   * the near queue holds vertices with tentative distance below
//     `threshold`; relax supersteps follow only their light edges, and an
//     improvement at or above the threshold goes to the far pile
//     (deduplicated per pile generation);
//   * when the near queue drains, every vertex of the bucket [bucket_lo,
//     threshold) has its final distance: one heavy superstep collects them
//     and relaxes their heavy edges once (all such relaxations land at or
//     above the threshold, in the far pile);
//   * one split pass then raises the threshold by delta and moves the far
//     vertices under it to the near queue.
// Heavy edges are thus relaxed once per reached vertex; only light edges can
// be relaxed again.  Supersteps run as one CUDA graph, as for BFS.
//
// Direction choice for the heavy step.  On scale-free graphs the first
// bucket settles the well-connected core, and its heavy out-edges are most
// of the graph's edges, while the vertices left unsettled are the periphery
// with few in-edges (RMAT-22 from the hub: 47.2 M heavy out-edges against
// 1.75 M in-edges of unsettled vertices).  The collect pass therefore also
// sums the heavy out-degree of the bucket and, over all buckets so far, the
// in-degree of the settled vertices; its last CTA picks a pull superstep
// when E - settled in-edges + V/2 (a dense pass reads about a vertex per two
// edges' worth of bytes) is below the heavy out-edge count.  The pull visits
// every vertex at or above the threshold and takes the minimum of dist[u] + w
// over its in-edges whose source is settled (dist[u] < threshold).  Every
// light edge of a settled vertex and every edge of an earlier bucket was
// relaxed already, so this minimum improves a vertex exactly where the push
// over the bucket's heavy edges would, and by the same value; each vertex is
// written by its own thread, and its new distance (at or above the
// threshold) does not pass the `dist[u] < threshold` filter of any reader.
//
// Around that: the solve runs on vertices renumbered by in-degree (the
// most-gathered distances share cache lines; one gather maps the result
// back), rows over sssp_hub_degree edges go to 256-edge warp pieces, a
// relax superstep skips an input vertex that it has already queued again,
// and a bucket is collected from the list of its relax inputs when that
// list is short.
//
// Buckets after the first (sssp_tail_delta > delta).  Past the first bucket
// the unsettled vertices are the periphery: low degree, mostly reached along
// one path.  There a bucket of width tail_delta relaxes every edge, light and
// heavy, in its relax supersteps and needs no heavy step, collect or bucket
// list: the relaxations are those of the narrow buckets (each vertex's edges
// about once; CPU replay at RMAT-22 from the hub: 1.67 M either way) in far
// fewer supersteps (37 -> 9 at width 256).  An improvement at or above the
// bucket's end still goes to the far pile, so the split and the result are
// those of delta-stepping with the wider bucket.
#include <algorithm>
#include <vector>

#include "olive_b200/olv_advance.cuh"
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"

namespace olv {

int traversal_workspace(olv_graph *g, bool pieces);
__global__ void k_fill_i32(int32_t *__restrict__ a, uint32_t n, int32_t x);

constexpr uint32_t kModeRelax = 0;
constexpr uint32_t kModeSplit = 2;
constexpr uint32_t kModeHeavy = 3;
constexpr uint32_t kModePull = 4;
constexpr uint32_t kModeSubSplit = 5;
constexpr uint32_t kModeRelaxAll = 6;   // relax every edge (buckets after the first, when wide)
// Default width of the first bucket.  With wide buckets after the first
// (sssp_tail_delta), a narrow first bucket is best on RMAT-24 from the hub
// (24: 1.90 ms; 16: 1.97; 32: 2.02; 48: 2.33; 64: 2.64): fewer light edges
// relaxed again inside it, the rest left to the pull and the wide buckets.
constexpr uint32_t kDefaultDelta = 24;

// Arrays the collect and pull passes read besides the queues.
struct SsspAux {
    const uint32_t *colptr;            // CSC row offsets
    const uint2 *crw;                  // CSC: (source, weight) per in-edge
    uint32_t vpull;                    // vertices [vpull, V) have no in-edges
    uint32_t vsplit;                   // the pull takes [vsplit, vpull) a thread per vertex
                                       // (renumbered: at most sssp_pull_split in-edges each)
    const uint2 *hdin;                 // per vertex: (heavy out-degree, in-degree)
    uint32_t *blist;                   // bucket list: the bucket's relax inputs, in order
    uint32_t *cmark;                   // bitmap: vertices collected so far this run
    uint32_t mark_words;               // words of one mark bitmap
    uint32_t bl_cap;                   // bucket list capacity (entries)
    unsigned long long E;
    int pull;                          // pull supersteps allowed
};

// Stable partition of every row into light (w <= delta) then heavy edges,
// written as (column, weight) pairs; one warp per row, two passes (count,
// then write in order).  Per vertex: rowmid (the split point) and its light
// and heavy ranges as uint2, so the advance reads a row's range with one load.
__global__ void k_partition_rows(const uint32_t *__restrict__ rowptr,
                                 const uint32_t *__restrict__ col, const uint32_t *__restrict__ w,
                                 uint32_t V, uint32_t delta, uint2 *__restrict__ pcw,
                                 uint32_t *__restrict__ rowmid, uint2 *__restrict__ lr,
                                 uint2 *__restrict__ hr) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (uint64_t u = warp; u < V; u += nwarps) {
        const uint32_t b = rowptr[u], e = rowptr[u + 1];
        uint32_t nl = 0;
        for (uint32_t base = b; base < e; base += 32) {
            const uint32_t i = base + lane;
            nl += __popc(__ballot_sync(0xffffffffu, i < e && w[i] <= delta));
        }
        uint32_t lo = b, hi = b + nl;
        for (uint32_t base = b; base < e; base += 32) {
            const uint32_t i = base + lane;
            const bool ok = i < e;
            const uint32_t wi = ok ? w[i] : 0, ci = ok ? col[i] : 0;
            const bool light = ok && wi <= delta;
            const unsigned ml = __ballot_sync(0xffffffffu, light);
            const unsigned mh = __ballot_sync(0xffffffffu, ok && !light);
            if (light)
                pcw[lo + __popc(ml & lt)] = make_uint2(ci, wi);
            else if (ok)
                pcw[hi + __popc(mh & lt)] = make_uint2(ci, wi);
            lo += __popc(ml);
            hi += __popc(mh);
        }
        if (lane == 0) {
            rowmid[u] = b + nl;
            lr[u] = make_uint2(b, b + nl);
            hr[u] = make_uint2(b + nl, e);
        }
    }
}

// In-edges as (source, weight) pairs for the pull superstep.
__global__ void k_pack_pairs(const uint32_t *__restrict__ a, const uint32_t *__restrict__ b,
                             unsigned long long n, uint2 *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = make_uint2(a[i], b[i]);
}

#ifndef OLV_SSSP_MINB
#define OLV_SSSP_MINB 3   // 3 CTAs per SM: up to 80 registers, no spills (4: 64, spills; 2% slower)
#endif
__device__ void sssp_end_step(TravCtl *c, cudaGraphConditionalHandle h, int use_cond,
                              uint32_t max_steps, uint32_t bl_cap);

struct SsspOp {
    static constexpr int kMinBlocks = OLV_SSSP_MINB;   // CTAs per SM the advance must fit
    static constexpr bool kEpilogue = true;   // the superstep's end step, when fused
    using SV = uint32_t;
    static constexpr bool kHasFar = true;
    static constexpr bool kPacked = true;   // (column, weight) pairs: one 8-byte load per edge
    // Dedupe bitmaps, 2 MB each at 16M vertices, so they stay in L2.  Near:
    // superstep t sets bits in nmark<t & 1> for the vertices it queues; those
    // vertices are superstep t+1's input queue, which clears them again
    // (on_input), so the bitmap is empty when superstep t+2 reuses it.  Far:
    // fmark<epoch & 1> holds the vertices of the current pile generation; the
    // split clears each pile entry's bit and sets the next generation's bit
    // for the entries it keeps.
    uint32_t *nmark0, *nmark1;
    uint32_t *fmark0, *fmark1;
    uint32_t *dist;
    uint32_t *nbits, *nprev, *fbits;
    uint32_t threshold, fmin;
    unsigned long long *relaxed_ctr;
    uint32_t *far_min;
    // end of the superstep run by the last CTA of the pieces kernel (instead
    // of a k_sssp_end launch) when end_fused is set
    cudaGraphConditionalHandle end_h;
    int end_fused, end_use_cond;
    uint32_t end_max_steps, end_bl_cap;
    __device__ __forceinline__ bool epilogue_on() const { return end_fused != 0; }
    __device__ __forceinline__ void epilogue(TravCtl *c) const {
        sssp_end_step(c, end_h, end_use_cond, end_max_steps, end_bl_cap);
    }

    __device__ __forceinline__ void begin(TravCtl *c) {
        dist = static_cast<uint32_t *>(c->vdata);
        const uint32_t stamp = c->steps + 1;
        nbits = (stamp & 1) ? nmark1 : nmark0;
        nprev = (stamp & 1) ? nmark0 : nmark1;
        fbits = (c->epoch & 1) ? fmark1 : fmark0;
        threshold = c->threshold;
        relaxed_ctr = &c->edges_relaxed;
        far_min = &c->far_min;
        fmin = 0xffffffffu;
    }
    struct Pre {
        uint32_t nd, cur;
    };
    __device__ __forceinline__ uint32_t src_value(uint32_t u) const { return __ldcg(&dist[u]); }
    __device__ __forceinline__ Pre prepare_packed(uint32_t du, uint32_t w, uint32_t v) const {
        uint32_t nd = du + w;
        if (nd < du || nd > (uint32_t)kInf) nd = (uint32_t)kInf;   // saturate
        return Pre{nd, __ldcg(&dist[v])};
    }
    // All of a thread's relaxations first, as reductions (no value returned, so
    // they pipeline), then one dedupe exchange per improved target, also all
    // issued before any result is used.  An edge counts as improving when its
    // candidate beats the distance loaded in prepare; a concurrent smaller
    // write makes the push redundant, never wrong: every decrease is made by a
    // thread that saw nd < dist and queues v (once per superstep through the
    // near mark, once per pile generation through the far mark), and a far
    // entry whose vertex ends up under the threshold is dropped by the split.
    template <int N>
    __device__ __forceinline__ void apply_n(const Pre (&p)[N], const uint32_t (&v)[N],
                                            int (&act)[N]) {
        bool cand[N];
#pragma unroll
        for (int j = 0; j < N; j++) {
            cand[j] = act[j] && p[j].nd < p[j].cur;
            if (cand[j]) atomicMin(&dist[v[j]], p[j].nd);
        }
        uint32_t old[N];
#pragma unroll
        for (int j = 0; j < N; j++) {
            old[j] = 0;
            if (cand[j]) {
                const uint32_t bit = 1u << (v[j] & 31);
                if (p[j].nd < threshold) {
                    old[j] = atomicOr(&nbits[v[j] >> 5], bit);
                } else {
                    fmin = p[j].nd < fmin ? p[j].nd : fmin;
                    old[j] = atomicOr(&fbits[v[j] >> 5], bit);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < N; j++) {
            const bool fresh = !((old[j] >> (v[j] & 31)) & 1u);
            if (!cand[j] || !fresh)
                act[j] = 0;
            else
                act[j] = p[j].nd < threshold ? 1 : 2;
        }
    }
    // The input vertex was queued (and marked) by the previous superstep.  If
    // this superstep has lowered its distance again, it is already queued for
    // the next one, which relaxes its edges from a distance no larger than
    // today's: expanding it now would only be repeated, so it is skipped.
    __device__ __forceinline__ bool on_input(uint32_t u) const {
        const uint32_t bit = 1u << (u & 31);
        atomicAnd(&nprev[u >> 5], ~bit);
        return !(__ldcg(&nbits[u >> 5]) & bit);
    }
    __device__ __forceinline__ void on_push(bool, uint32_t) {}
    __device__ __forceinline__ void flush(unsigned long long relaxed) {
        warp_add64(relaxed, relaxed_ctr);
        const uint32_t m = __reduce_min_sync(0xffffffffu, fmin);
        if (lane_id() == 0 && m != 0xffffffffu) atomicMin(far_min, m);
    }
};

__device__ void sssp_begin(TravCtl *c);

__global__ void k_sssp_init(TravCtl *c, uint32_t *dist, uint32_t *q0, uint32_t src,
                            uint32_t delta, uint32_t sub, uint32_t sub_buckets,
                            uint32_t tail_width, uint32_t route, uint32_t direct_min,
                            const uint32_t *newid) {
    if (newid) src = newid[src];   // relabelled run: the source's new id
    TravCtl t = {};
    t.qsize[0] = 1;
    t.vdata = dist;
    t.delta = delta;
    t.bucket_end = delta;
    t.sub_width = sub < delta ? sub : 0;
    t.sub_buckets = sub_buckets;
    t.heavy_index = 0;
    t.tail_width = tail_width > delta ? tail_width : 0;
    t.all_edges = 0;
    t.route = t.tail_width != 0 && route;
    t.direct_min = t.route ? direct_min : 0;
    t.threshold = (t.sub_width && sub_buckets > 0) ? t.sub_width : delta;
    t.epoch = 1;
    t.far_min = 0xffffffffu;
    t.heavy_done = 0;
    t.bucket_lo = 0;
    *c = t;
    dist[src] = 0;
    q0[0] = src;
    sssp_begin(c);
}

static __device__ __forceinline__ uint32_t sat_add(uint32_t a, uint32_t b) {
    const uint64_t t = (uint64_t)a + b;
    return t > (uint64_t)kInf ? (uint32_t)kInf : (uint32_t)t;
}

// Choose the next superstep's mode and reset its counters:
//   relax      the near queue is not empty: relax its light edges;
//   sub-split  inside a heavy bucket [bucket_lo, bucket_end) whose light
//              phase runs in sub-buckets of sub_width: when the near queue of
//              one sub-bucket drains, every vertex under the threshold is
//              final (light edges of later vertices land at or above it, heavy
//              edges past bucket_end), so the far pile is split at the next
//              sub-bucket's end; the bucket list and the pending heavy step
//              carry over;
//   heavy      the heavy bucket is settled: collect it and relax its heavy
//              edges (or pull them);
//   split      start the next heavy bucket at max(threshold, far minimum).
__device__ void sssp_begin(TravCtl *c) {
    if (c->done) return;
    if (c->qsize[c->cur] > 0) {
        c->mode = c->all_edges ? kModeRelaxAll : kModeRelax;
        c->qsize[c->cur ^ 1] = 0;
        c->npieces = 0;
        return;
    }
    if (!c->heavy_done && c->threshold < c->bucket_end && c->far_size[c->far_cur] > 0 &&
        c->far_min < c->bucket_end) {
        c->mode = kModeSubSplit;
        c->split_lo = c->threshold;   // far entries below it were settled already
        const uint32_t lo = c->threshold > c->far_min ? c->threshold : c->far_min;
        const uint32_t t = sat_add(lo, c->sub_width);
        c->threshold = t < c->bucket_end ? t : c->bucket_end;
        c->far_size[c->far_cur ^ 1] = 0;
        c->far_min = 0xffffffffu;
        return;
    }
    if (!c->heavy_done) {   // bucket settled: collect it and relax its heavy edges
        // a large first bucket (its relax inputs listed) goes straight to the
        // pull: on a scale-free graph its heavy out-edges far outnumber the
        // unsettled vertices' in-edges, and with wide buckets after it no
        // later heavy step needs the collect's sums
        if (!c->pull_pending && c->direct_min && c->heavy_index == 0 &&
            (c->bl_over || c->bl_size >= c->direct_min))
            c->pull_pending = 1;
        c->mode = c->pull_pending ? kModePull : kModeHeavy;
        c->qsize[c->cur] = 0;
        c->qsize[c->cur ^ 1] = 0;
        c->npieces = 0;
        c->heavy_work = 0;
        c->aux_done = 0;
        if (c->mode == kModePull && c->route) {   // a routing pull refills the far pile
            c->far_size[c->far_cur ^ 1] = 0;
            c->far_min = 0xffffffffu;
        }
        return;
    }
    if (c->far_size[c->far_cur] == 0) {
        c->done = 1;
        return;
    }
    // next heavy bucket starts at max(threshold, smallest far distance)
    c->mode = kModeSplit;
    c->split_lo = c->threshold;   // far entries below it were settled already
    c->bucket_lo = c->threshold;
    const uint32_t lo = c->threshold > c->far_min ? c->threshold : c->far_min;
    c->heavy_index++;
    c->all_edges = c->tail_width != 0;   // buckets after the first: wide, every edge
    const uint32_t width = c->all_edges ? c->tail_width : c->delta;
    c->bucket_end = sat_add(lo, width);
    const bool sub = !c->all_edges && c->sub_width && c->heavy_index < c->sub_buckets;
    const uint32_t t = sat_add(lo, sub ? c->sub_width : width);
    c->threshold = t < c->bucket_end ? t : c->bucket_end;
    c->far_size[c->far_cur ^ 1] = 0;
    c->far_min = 0xffffffffu;
}


// The two far-pile generation bitmaps (kernel argument by value).
struct FarMarks {
    uint32_t *m0, *m1;
};

// Per-warp staging of queue appends in shared memory (one buffer per warp and
// output list), flushed to the global list with one atomic per flush.
struct WarpStage {
    uint32_t *buf, *n, *lim;
    __device__ __forceinline__ void init() {
        if (lane_id() == 0) {
            *n = 0;
            *lim = kWarpStage;
        }
        __syncwarp();
    }
    // make room for up to `room` entries (warp-uniform)
    __device__ __forceinline__ void reserve(uint32_t room, uint32_t *q, uint32_t *qsize) {
        __syncwarp();
        if (*n + room > kWarpStage) warp_stage_flush(buf, n, lim, q, qsize);
    }
};

// Heavy superstep, step 1: the vertices of the settled bucket
// [bucket_lo, threshold) become the input queue.  Every such vertex was the
// input of one of the bucket's relax supersteps (it entered the bucket from
// the far pile through the split, or by a light relaxation), so when the
// bucket list (those inputs, kept by the aux pass) is short, the collect
// reads the list, dropping repeats with a bitmap of the vertices collected so
// far in the run (a vertex is collected once: later buckets start above its
// distance); otherwise it reads every vertex's distance, four per thread.
// With pull supersteps allowed, the collected vertices' heavy out-degrees and
// in-degrees are summed into heavy_work and settled_in for the direction
// choice.
__device__ void sssp_collect(uint32_t V, TravCtl *c, uint32_t *q0, uint32_t *q1,
                             const SsspAux &x, WarpStage st) {
    unsigned long long hw = 0, si = 0;
    const uint32_t *dist = static_cast<const uint32_t *>(c->vdata);
    const uint32_t lo = c->bucket_lo, hi = c->threshold;
    uint32_t *q = c->cur ? q1 : q0;
    uint32_t *qsize = &c->qsize[c->cur];
    const uint32_t nl = c->bl_size;
    const bool from_list = !c->bl_over && (uint64_t)nl * 8 < V;
    const uint64_t nquad = from_list ? ((uint64_t)nl + 3) / 4 : ((uint64_t)V + 3) / 4;
    const bool vec = ((uintptr_t)dist & 15) == 0;
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < nquad;
         base += (uint64_t)gridDim.x * kBlock) {
        int act[4];
        uint32_t vv[4];
        uint32_t d[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
        if (from_list) {   // entries base*4 + j*kBlock + t: coalesced per j
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint64_t i = base * 4 + (uint64_t)j * kBlock + threadIdx.x;
                vv[j] = i < nl ? x.blist[i] : 0u;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint64_t i = base * 4 + (uint64_t)j * kBlock + threadIdx.x;
                if (i < nl) d[j] = __ldcg(dist + vv[j]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                act[j] = d[j] >= lo && d[j] < hi;
                if (act[j]) {
                    const uint32_t bit = 1u << (vv[j] & 31);
                    if (atomicOr(&x.cmark[vv[j] >> 5], bit) & bit) act[j] = 0;   // a repeat
                }
            }
        } else {
            const uint64_t v0 = (base + threadIdx.x) * 4;
            if (vec && v0 + 3 < V) {
                const uint4 d4 = __ldcg(reinterpret_cast<const uint4 *>(dist + v0));
                d[0] = d4.x;
                d[1] = d4.y;
                d[2] = d4.z;
                d[3] = d4.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (v0 + j < V) d[j] = __ldcg(dist + v0 + j);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                act[j] = d[j] >= lo && d[j] < hi;   // vertices >= V hold 0xffffffff
                vv[j] = (uint32_t)(v0 + j);
            }
        }
        if (x.pull) {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (act[j]) {
                    const uint2 h = x.hdin[vv[j]];
                    hw += h.x;
                    si += h.y;
                }
        }
        st.reserve(32 * 4, q, qsize);
        stage_push_n<4>(act, vv, 1, st.buf, st.n, st.lim, kWarpStage, q, qsize);
    }
    warp_stage_flush(st.buf, st.n, st.lim, q, qsize);
    if (x.pull) {
        warp_add64(hw, &c->heavy_work);
        warp_add64(si, &c->settled_in);
    }
}

// The collect pass's last CTA to finish chooses push or pull for the heavy
// edges of the bucket (all CTAs' sums are in by then: each CTA fences its
// atomics before counting itself done).  Pull empties the collected queue,
// so the push kernels of this superstep find no work, and marks the pull
// superstep to follow.
__device__ void sssp_choose(uint32_t V, TravCtl *c, const SsspAux &x) {
    __shared__ uint32_t s_last;
    __threadfence();   // this thread's sums are visible before the CTA counts itself done
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&c->aux_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    const unsigned long long hw = atomicAdd(&c->heavy_work, 0ull);
    const unsigned long long si = atomicAdd(&c->settled_in, 0ull);
    const unsigned long long pull_edges = (x.E > si ? x.E - si : 0ull) + V / 2;
    if (pull_edges < hw) {
        c->pull_pending = 1;
        c->qsize[c->cur] = 0;
    }
}

// Relaxation candidate of in-edge i: dist[u] + w when u is settled
// (dist[u] < hi), else no candidate.
__device__ __forceinline__ uint32_t pull_cand(uint32_t du, uint32_t w, uint32_t hi) {
    if (du >= hi) return 0xffffffffu;
    uint32_t nd = du + w;
    if (nd < du || nd > (uint32_t)kInf) nd = (uint32_t)kInf;   // saturate
    return nd;
}

// One pulled vertex v with old distance d and pull minimum best (<= d): the
// push action (0 none, 1 near queue, 2 far pile).  Without routing an
// improvement goes to the far pile once per generation (fbits); with it every
// vertex at or above the threshold with a finite distance goes to the near
// queue of the next bucket (under nend) or to the next generation (fnext).
__device__ __forceinline__ int pull_out(uint32_t best, uint32_t d, uint32_t v, uint32_t hi,
                                        bool route, uint32_t nend, uint32_t *dist,
                                        uint32_t *fbits, uint32_t *fnext, uint32_t &fmin) {
    const uint32_t bit = 1u << (v & 31);
    if (best < d) dist[v] = best;
    if (!route) {
        if (best >= d) return 0;   // only vertices at or above the threshold can improve
        fmin = best < fmin ? best : fmin;
        return (atomicOr(&fbits[v >> 5], bit) & bit) ? 0 : 2;
    }
    if (d < hi || best >= (uint32_t)kInf) return 0;   // settled, or unreached
    if (best < nend) return 1;
    atomicOr(&fnext[v >> 5], bit);
    fmin = best < fmin ? best : fmin;
    return 2;
}

// Pull superstep: every vertex at or above the threshold takes the minimum
// candidate over its in-edges; improved vertices go to the far pile (once
// per pile generation).  Each CTA iteration covers 1024 vertices, four per
// thread (16-byte distance and column-pointer loads); the chunk's in-degrees
// are scanned across the CTA, its threads then take the chunk's in-edges in
// order, kPullItems per thread in flight (owner vertex by binary search over
// the scan), and fold candidates into a shared per-vertex minimum.
constexpr int kPullItems = 4;
constexpr uint32_t kPullChunk = 4 * kBlock;
//
// Routing (buckets after the first are wide and relax every edge): the pull
// also opens the next bucket, [threshold, threshold + tail_width), itself.
// Every vertex it visits with a finite distance goes to the near queue of
// that bucket or, at or above its end, to the far pile's next generation
// (marks set; the visits cover every vertex that can hold a distance, so the
// old pile, whose marks are cleared word by word, is dropped), and no split
// pass follows.
__device__ void sssp_pull(uint32_t V, TravCtl *c, uint32_t *q0, uint32_t *q1, uint32_t *far0,
                          uint32_t *far1, FarMarks fm, const SsspAux &x, WarpStage sn,
                          WarpStage sf) {
    uint32_t *dist = static_cast<uint32_t *>(c->vdata);
    const uint32_t hi = c->threshold;
    const bool route = c->route != 0;
    const uint32_t nend = route ? sat_add(hi, c->tail_width) : 0;   // end of the next bucket
    uint32_t *fbits = (c->epoch & 1) ? fm.m1 : fm.m0;
    uint32_t *fnext = (c->epoch & 1) ? fm.m0 : fm.m1;
    // routing fills the other far buffer (the next generation)
    uint32_t *far = (c->far_cur ^ (route ? 1u : 0u)) ? far1 : far0;
    uint32_t *far_size = &c->far_size[c->far_cur ^ (route ? 1u : 0u)];
    uint32_t *qn = c->cur ? q1 : q0;
    uint32_t *qn_size = &c->qsize[c->cur];
    __shared__ uint32_t s_off[kPullChunk + 1], s_beg[kPullChunk], s_best[kPullChunk], s_warp[33];
    const bool vec = ((uintptr_t)dist & 15) == 0 && ((uintptr_t)x.colptr & 15) == 0;
    const uint32_t lane = lane_id();
    uint32_t fmin = 0xffffffffu;
    unsigned long long scanned = 0;
    // vertices past vpull have no in-edges (the renumbered ids put them
    // last); [vsplit, vpull) go a thread per vertex below
    for (uint64_t base = (uint64_t)blockIdx.x * kPullChunk; base < x.vsplit;
         base += (uint64_t)gridDim.x * kPullChunk) {
        const uint64_t v0 = base + 4 * (uint64_t)threadIdx.x;
        uint32_t d[4] = {0u, 0u, 0u, 0u}, b[4] = {0u, 0u, 0u, 0u}, e[4] = {0u, 0u, 0u, 0u};
        if (vec && v0 + 4 <= V) {
            const uint4 d4 = __ldcg(reinterpret_cast<const uint4 *>(dist + v0));
            d[0] = d4.x;
            d[1] = d4.y;
            d[2] = d4.z;
            d[3] = d4.w;
            if (d[0] >= hi || d[1] >= hi || d[2] >= hi || d[3] >= hi) {
                const uint4 c4 = *reinterpret_cast<const uint4 *>(x.colptr + v0);
                const uint32_t c5 = x.colptr[v0 + 4];
                if (d[0] >= hi) { b[0] = c4.x; e[0] = c4.y; }
                if (d[1] >= hi) { b[1] = c4.y; e[1] = c4.z; }
                if (d[2] >= hi) { b[2] = c4.z; e[2] = c4.w; }
                if (d[3] >= hi) { b[3] = c4.w; e[3] = c5; }
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (v0 + j < V) {
                    d[j] = __ldcg(dist + v0 + j);
                    if (d[j] >= hi) {
                        b[j] = x.colptr[v0 + j];
                        e[j] = x.colptr[v0 + j + 1];
                    }
                }
        }
        // vertices past V keep d = 0 < hi and no in-edges
        const uint32_t t01 = (e[0] - b[0]) + (e[1] - b[1]);
        const uint32_t t = t01 + (e[2] - b[2]) + (e[3] - b[3]);
        uint32_t total;
        const uint32_t off = block_exclusive_scan(t, &total, s_warp);
        const uint32_t r0 = 4 * threadIdx.x;
        s_off[r0] = off;
        s_off[r0 + 1] = off + (e[0] - b[0]);
        s_off[r0 + 2] = off + t01;
        s_off[r0 + 3] = off + t01 + (e[2] - b[2]);
        if (threadIdx.x == kBlock - 1) s_off[kPullChunk] = total;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            s_beg[r0 + j] = b[j];
            s_best[r0 + j] = d[j];
        }
        __syncthreads();
        for (uint32_t k0 = threadIdx.x; k0 < total; k0 += kBlock * kPullItems) {
            uint32_t own[kPullItems], u[kPullItems], w[kPullItems], du[kPullItems];
#pragma unroll
            for (int j = 0; j < kPullItems; j++) {
                const uint32_t k = k0 + j * kBlock;
                own[j] = kPullChunk;
                u[j] = 0;
                w[j] = 0;
                if (k < total) {
                    uint32_t lo = 0;   // last vertex with s_off[vertex] <= k
#pragma unroll
                    for (uint32_t step = kPullChunk / 2; step > 0; step >>= 1)
                        if (s_off[lo + step] <= k) lo += step;
                    own[j] = lo;
                    const uint32_t i = s_beg[lo] + (k - s_off[lo]);
                    const uint2 t = x.crw[i];
                    u[j] = t.x;
                    w[j] = t.y;
                }
            }
#pragma unroll
            for (int j = 0; j < kPullItems; j++)
                du[j] = own[j] < kPullChunk ? __ldcg(&dist[u[j]]) : 0xffffffffu;
#pragma unroll
            for (int j = 0; j < kPullItems; j++) {
                if (own[j] < kPullChunk) {
                    const uint32_t nd = pull_cand(du[j], w[j], hi);
                    if (nd < s_best[own[j]]) atomicMin(&s_best[own[j]], nd);
                }
            }
        }
        __syncthreads();
        scanned += t;
        if (route && threadIdx.x < kPullChunk / 32 && base / 32 + threadIdx.x < x.mark_words)
            fbits[base / 32 + threadIdx.x] = 0;   // the old pile's marks of this chunk
        int act[4];
        uint32_t va[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            va[j] = (uint32_t)(v0 + j);
            act[j] = pull_out(s_best[r0 + j], d[j], va[j], hi, route, nend, dist, fbits, fnext,
                              fmin);
        }
        sn.reserve(32 * 4, qn, qn_size);
        stage_push_n<4>(act, va, 1, sn.buf, sn.n, sn.lim, kWarpStage, qn, qn_size);
        sf.reserve(32 * 4, far, far_size);
        stage_push_n<4>(act, va, 2, sf.buf, sf.n, sf.lim, kWarpStage, far, far_size);
        __syncthreads();   // s_off / s_beg / s_best are rewritten by the next chunk
    }
    // Short rows (renumbered suffix, at most sssp_pull_split in-edges each): a
    // thread takes four consecutive vertices and scans the in-edges of the
    // unsettled ones itself, four in flight; no shared memory or barriers.
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock * 4 + x.vsplit; base < x.vpull;
         base += (uint64_t)gridDim.x * kBlock * 4) {
        const uint64_t v0 = base + 4 * (uint64_t)threadIdx.x;
        uint32_t d[4] = {0u, 0u, 0u, 0u}, b[4] = {0u, 0u, 0u, 0u}, e[4] = {0u, 0u, 0u, 0u};
        if (vec && v0 + 4 <= V) {
            const uint4 d4 = __ldcg(reinterpret_cast<const uint4 *>(dist + v0));
            d[0] = d4.x;
            d[1] = d4.y;
            d[2] = d4.z;
            d[3] = d4.w;
            if (d[0] >= hi || d[1] >= hi || d[2] >= hi || d[3] >= hi) {
                const uint4 c4 = *reinterpret_cast<const uint4 *>(x.colptr + v0);
                const uint32_t c5 = x.colptr[v0 + 4];
                if (d[0] >= hi) { b[0] = c4.x; e[0] = c4.y; }
                if (d[1] >= hi) { b[1] = c4.y; e[1] = c4.z; }
                if (d[2] >= hi) { b[2] = c4.z; e[2] = c4.w; }
                if (d[3] >= hi) { b[3] = c4.w; e[3] = c5; }
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (v0 + j < V) {
                    d[j] = __ldcg(dist + v0 + j);
                    if (d[j] >= hi) {
                        b[j] = x.colptr[v0 + j];
                        e[j] = x.colptr[v0 + j + 1];
                    }
                }
        }
        // the four vertices' in-edges are read in step, four per vertex per
        // round (at most two rounds), so sixteen loads (and then sixteen
        // gathers) are in flight
        uint32_t best[4], len = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            best[j] = d[j];
            scanned += e[j] - b[j];
            len = max(len, e[j] - b[j]);
        }
        for (uint32_t o = 0; o < len; o += 4) {
            uint2 t[4][4];
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int k = 0; k < 4; k++)
                    t[j][k] = b[j] + o + k < e[j] ? x.crw[b[j] + o + k] : make_uint2(0u, 0u);
            uint32_t du[4][4];
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int k = 0; k < 4; k++)
                    du[j][k] = b[j] + o + k < e[j] ? __ldcg(&dist[t[j][k].x]) : 0xffffffffu;
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int k = 0; k < 4; k++) best[j] = min(best[j], pull_cand(du[j][k], t[j][k].y, hi));
        }
        if (route && threadIdx.x < kBlock * 4 / 32 && base / 32 + threadIdx.x < x.mark_words)
            fbits[base / 32 + threadIdx.x] = 0;   // the old pile's marks of these vertices
        int act[4];
        uint32_t va[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            va[j] = (uint32_t)(v0 + j);
            act[j] = pull_out(best[j], d[j], va[j], hi, route, nend, dist, fbits, fnext, fmin);
        }
        sn.reserve(32 * 4, qn, qn_size);
        stage_push_n<4>(act, va, 1, sn.buf, sn.n, sn.lim, kWarpStage, qn, qn_size);
        sf.reserve(32 * 4, far, far_size);
        stage_push_n<4>(act, va, 2, sf.buf, sf.n, sf.lim, kWarpStage, far, far_size);
    }
    warp_stage_flush(sn.buf, sn.n, sn.lim, qn, qn_size);
    warp_stage_flush(sf.buf, sf.n, sf.lim, far, far_size);
    const uint32_t m = __reduce_min_sync(0xffffffffu, fmin);
    if (lane == 0 && m != 0xffffffffu) atomicMin(&c->far_min, m);
    warp_add64(scanned, &c->edges_relaxed);
}

// Split the far pile: stale entries (distance below the old threshold) are
// dropped, entries under the new threshold become the near queue, the rest
// move to the other far buffer under the next generation.
__device__ void sssp_split(TravCtl *c, uint32_t *q0, uint32_t *q1, uint32_t *far0,
                           uint32_t *far1, FarMarks fm, WarpStage sn, WarpStage sf) {
    const uint32_t *dist = static_cast<const uint32_t *>(c->vdata);
    const uint32_t fc = c->far_cur;
    const uint32_t n = c->far_size[fc];
    const uint32_t *fin = fc ? far1 : far0;
    uint32_t *fout = fc ? far0 : far1;
    uint32_t *fout_size = &c->far_size[fc ^ 1];
    uint32_t *qn = c->cur ? q1 : q0;
    uint32_t *qn_size = &c->qsize[c->cur];
    const uint32_t lo = c->split_lo, hi = c->threshold;
    uint32_t *fcur = (c->epoch & 1) ? fm.m1 : fm.m0;
    uint32_t *fnext = (c->epoch & 1) ? fm.m0 : fm.m1;
    uint32_t fmin = 0xffffffffu;
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < n;
         base += (uint64_t)gridDim.x * kBlock) {
        const uint64_t i = base + threadIdx.x;
        int act[1] = {0};
        uint32_t v[1] = {0};
        if (i < n) {
            v[0] = fin[i];
            const uint32_t bit = 1u << (v[0] & 31);
            atomicAnd(&fcur[v[0] >> 5], ~bit);   // this generation's pile is consumed
            const uint32_t d = __ldcg(&dist[v[0]]);
            if (d >= lo) {
                if (d < hi) {
                    act[0] = 1;
                } else {
                    act[0] = 2;
                    atomicOr(&fnext[v[0] >> 5], bit);
                    fmin = d < fmin ? d : fmin;
                }
            }
        }
        sn.reserve(32, qn, qn_size);
        stage_push_n<1>(act, v, 1, sn.buf, sn.n, sn.lim, kWarpStage, qn, qn_size);
        sf.reserve(32, fout, fout_size);
        stage_push_n<1>(act, v, 2, sf.buf, sf.n, sf.lim, kWarpStage, fout, fout_size);
    }
    warp_stage_flush(sn.buf, sn.n, sn.lim, qn, qn_size);
    warp_stage_flush(sf.buf, sf.n, sf.lim, fout, fout_size);
    const uint32_t m = __reduce_min_sync(0xffffffffu, fmin);
    if (lane_id() == 0 && m != 0xffffffffu) atomicMin(&c->far_min, m);
}

// End of a superstep (one thread): account for what it did, decide whether
// the run is over, set the next superstep's mode, and tell the enclosing
// while-conditional graph whether to run another.
__device__ void sssp_end_step(TravCtl *c, cudaGraphConditionalHandle h, int use_cond,
                              uint32_t max_steps, uint32_t bl_cap) {
    if (!c->done) {
        if (c->mode == kModeRelax) {
            // the aux pass appended this superstep's input to the bucket list
            // under the same capacity test
            const uint32_t n = c->qsize[c->cur];
            if (!c->bl_over) {
                if ((uint64_t)c->bl_size + n <= bl_cap)
                    c->bl_size += n;
                else
                    c->bl_over = 1;
            }
            c->cur ^= 1;
        } else if (c->mode == kModeRelaxAll) {
            c->cur ^= 1;   // no bucket list: an all-edge bucket has no heavy step
        } else if (c->mode == kModeHeavy) {
            c->qsize[c->cur] = 0;
            c->heavy_done = c->pull_pending ? 0 : 1;   // pending: the pull superstep is next
        } else if (c->mode == kModePull) {
            c->pull_pending = 0;
            c->heavy_done = 1;
            c->pull_steps++;
            if (c->route) {   // the pull routed every vertex: the next bucket is open
                c->bucket_lo = c->threshold;
                c->heavy_index++;
                c->all_edges = 1;
                c->threshold = c->bucket_end = sat_add(c->threshold, c->tail_width);
                c->far_cur ^= 1;
                c->epoch++;
                c->bl_size = 0;
                c->bl_over = 0;
            }
        } else if (c->mode == kModeSubSplit) {
            c->far_cur ^= 1;   // the bucket list and the pending heavy step carry over
            c->epoch++;
        } else {
            c->bl_size = 0;   // a new bucket: its list starts empty
            c->bl_over = 0;
            c->far_cur ^= 1;
            c->epoch++;
            c->heavy_done = c->all_edges ? 1 : 0;   // all-edge buckets: nothing left after relax
        }
        c->steps++;
        if (c->qsize[c->cur] == 0 && c->far_size[c->far_cur] == 0 && c->heavy_done) c->done = 1;
        if (c->steps > max_steps) {
            c->err = 2;
            c->done = 1;
        }
        sssp_begin(c);   // mode and counters of the next superstep
    }
    if (use_cond) cudaGraphSetConditional(h, c->done ? 0u : 1u);
}

__global__ void k_sssp_end(TravCtl *c, cudaGraphConditionalHandle h, int use_cond,
                           uint32_t max_steps, uint32_t bl_cap) {
    sssp_end_step(c, h, use_cond, max_steps, bl_cap);
}

// The superstep's dense pass: collect the settled bucket (heavy mode), pull
// over the unsettled vertices' in-edges (pull mode) or split the far pile
// (split mode); nothing in relax mode.
__global__ void __launch_bounds__(kBlock)
k_sssp_aux(uint32_t V, TravCtl *c, uint32_t *q0, uint32_t *q1, uint32_t *far0, uint32_t *far1,
           FarMarks fm, SsspAux x) {
    if (c->done) return;
    const uint32_t mode = c->mode;
    if (mode == kModeRelax) {   // append this superstep's input to the bucket list
        const uint32_t n = c->qsize[c->cur];
        if (c->bl_over || (uint64_t)c->bl_size + n > x.bl_cap) return;   // k_sssp_end: overflow
        const uint32_t *qin = c->cur ? q1 : q0;
        uint32_t *dst = x.blist + c->bl_size;
        for (uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x; i < n;
             i += (uint64_t)gridDim.x * kBlock)
            dst[i] = qin[i];
        return;
    }
    if (mode != kModeHeavy && mode != kModeSplit && mode != kModePull && mode != kModeSubSplit)
        return;
    __shared__ uint32_t s_a[kBlock / 32][kWarpStage], s_b[kBlock / 32][kWarpStage];
    __shared__ uint32_t s_an[kBlock / 32], s_alim[kBlock / 32];
    __shared__ uint32_t s_bn[kBlock / 32], s_blim[kBlock / 32];
    const uint32_t wl = threadIdx.x >> 5;
    WarpStage sa{s_a[wl], &s_an[wl], &s_alim[wl]};
    WarpStage sb{s_b[wl], &s_bn[wl], &s_blim[wl]};
    sa.init();
    sb.init();
    if (mode == kModeHeavy) {
        sssp_collect(V, c, q0, q1, x, sa);
        if (x.pull) sssp_choose(V, c, x);
    } else if (mode == kModePull) {
        sssp_pull(V, c, q0, q1, far0, far1, fm, x, sa, sb);
    } else {
        sssp_split(c, q0, q1, far0, far1, fm, sa, sb);
    }
}

// Sum of out-degrees and count of reached vertices (the GTEPS basis).
__global__ void k_reached_edges(const uint32_t *__restrict__ rowptr,
                                const uint32_t *__restrict__ dist, uint32_t V,
                                unsigned long long *out /*[2]*/) {
    unsigned long long e = 0, n = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x)
        if (dist[v] != (uint32_t)kInf) {
            e += rowptr[v + 1] - rowptr[v];
            n++;
        }
    warp_add64(e, &out[0]);
    warp_add64(n, &out[1]);
}

// ------------------------------------------------------------------ host --
// words of one dedupe bitmap (rounded up to 64 words = 256 bytes)
static size_t mark_words(uint32_t V) { return (((size_t)V + 31) / 32 + 63) & ~(size_t)63; }
// bitmaps: near marks x2, far-pile generation marks x2, collected vertices
constexpr size_t kMarks = 5;

static uint32_t sssp_delta(olv_graph *g) {
    if (g->tune.sssp_delta) return g->tune.sssp_delta;
    return kDefaultDelta;
}

// Per vertex (heavy out-degree, in-degree): what the collect pass sums for the
// push/pull choice, one 8-byte load per collected vertex.
__global__ void k_heavy_in_degrees(const uint32_t *__restrict__ rowptr,
                                   const uint32_t *__restrict__ rowmid,
                                   const uint32_t *__restrict__ colptr, uint32_t V,
                                   uint2 *__restrict__ hdin) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x)
        hdin[v] = make_uint2(rowptr[v + 1] - rowmid[v], colptr[v + 1] - colptr[v]);
}

// Row i of the renumbered structure is row perm[i] of the old one, its
// entries in the same order, neighbour ids mapped through newid, weights
// carried along.  One warp per row.
__global__ void k_sssp_relabel(const uint32_t *__restrict__ old_ptr,
                               const uint32_t *__restrict__ old_idx,
                               const uint32_t *__restrict__ old_w,
                               const uint32_t *__restrict__ perm,
                               const uint32_t *__restrict__ newid,
                               const uint32_t *__restrict__ new_ptr, uint32_t n,
                               uint32_t *__restrict__ new_idx, uint32_t *__restrict__ new_w) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w; i < n; i += nw) {
        const uint32_t v = perm[i];
        const uint32_t b = old_ptr[v], e = old_ptr[v + 1], o = new_ptr[i];
        for (uint32_t k = lane; k < e - b; k += 32) {
            new_idx[o + k] = newid[old_idx[b + k]];
            new_w[o + k] = old_w[b + k];
        }
    }
}

// Distances back to the caller's ids: out[v] = dnew[newid[v]].
// Distances back to the caller's ids; with red, also the sum of out-degrees
// and the count of the reached vertices (k_reached_edges in the same pass).
// Four vertices per thread, their four gathers in flight (the gather of the
// renumbered distances is the pass's latency).
__global__ void k_sssp_unrelabel(const uint32_t *__restrict__ dnew,
                                 const uint32_t *__restrict__ newid, uint32_t V,
                                 uint32_t *__restrict__ out, const uint32_t *__restrict__ rowptr,
                                 unsigned long long *red /*[2] or null*/) {
    unsigned long long e = 0, n = 0;
    const bool vec = (((uintptr_t)newid | (uintptr_t)out | (uintptr_t)rowptr) & 15) == 0;
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; 4 * q < V;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v0 = 4 * q;
        uint32_t d[4];
        if (vec && v0 + 4 <= V) {
            const uint4 k4 = *reinterpret_cast<const uint4 *>(newid + v0);
            d[0] = __ldg(&dnew[k4.x]);
            d[1] = __ldg(&dnew[k4.y]);
            d[2] = __ldg(&dnew[k4.z]);
            d[3] = __ldg(&dnew[k4.w]);
            *reinterpret_cast<uint4 *>(out + v0) = make_uint4(d[0], d[1], d[2], d[3]);
            if (red) {
                const uint4 r4 = *reinterpret_cast<const uint4 *>(rowptr + v0);
                const uint32_t r5 = rowptr[v0 + 4];
                const uint32_t dg[4] = {r4.y - r4.x, r4.z - r4.y, r4.w - r4.z, r5 - r4.w};
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (d[j] != (uint32_t)kInf) {
                        e += dg[j];
                        n++;
                    }
            }
        } else {
            for (uint64_t v = v0; v < V && v < v0 + 4; v++) {
                const uint32_t dv = __ldg(&dnew[newid[v]]);
                out[v] = dv;
                if (red && dv != (uint32_t)kInf) {
                    e += rowptr[v + 1] - rowptr[v];
                    n++;
                }
            }
        }
    }
    if (red) {
        warp_add64(e, &red[0]);
        warp_add64(n, &red[1]);
    }
}

// Renumber the vertices by in-degree, highest first (a stable counting sort
// on the host, once per graph), and build the CSR and CSC with weights in
// the new ids.  The relax supersteps gather the distances of edge targets;
// on a scale-free graph most gathers hit the high in-degree vertices, whose
// distances then share cache lines instead of one 32-byte sector each.
static int sssp_relabel(olv_graph *g) {
    Workspace &ws = g->ws;
    if (ws.sr_built) return OLV_OK;
    const uint32_t V = g->V;
    const uint64_t E = g->E;
    cudaStream_t s = g->stream;
    std::vector<uint32_t> rp((size_t)V + 1), cp((size_t)V + 1);
    OLV_CUDA(cudaMemcpyAsync(rp.data(), g->rowptr.p, ((size_t)V + 1) * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaMemcpyAsync(cp.data(), g->colptr.p, ((size_t)V + 1) * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    uint32_t maxd = 0;
    for (uint32_t v = 0; v < V; v++) maxd = std::max(maxd, cp[v + 1] - cp[v]);
    std::vector<uint64_t> start((size_t)maxd + 2, 0);
    for (uint32_t v = 0; v < V; v++) start[maxd - (cp[v + 1] - cp[v]) + 1]++;
    for (size_t d = 1; d < start.size(); d++) start[d] += start[d - 1];
    std::vector<uint32_t> perm(V), newid(V), nrp((size_t)V + 1), ncp((size_t)V + 1);
    for (uint32_t v = 0; v < V; v++) {
        const uint32_t i = (uint32_t)start[maxd - (cp[v + 1] - cp[v])]++;
        perm[i] = v;
        newid[v] = i;
    }
    // in-degree > 0, and > 4, 8, 16, 32 (the pull's short-row bounds):
    // prefixes of the new numbering
    uint32_t vnz = 0, vlong[4] = {0, 0, 0, 0};
    for (uint32_t v = 0; v < V; v++) {
        const uint32_t din = cp[v + 1] - cp[v];
        vnz += din != 0;
        for (int k = 0; k < 4; k++) vlong[k] += din > (4u << k);
    }
    ws.sr_vnz = vnz;
    for (int k = 0; k < 4; k++) ws.sr_vlong[k] = vlong[k];
    nrp[0] = 0;
    ncp[0] = 0;
    for (uint32_t i = 0; i < V; i++) {
        nrp[i + 1] = nrp[i] + (rp[perm[i] + 1] - rp[perm[i]]);
        ncp[i + 1] = ncp[i] + (cp[perm[i] + 1] - cp[perm[i]]);
    }
    OLV_TRY(ws.sr_perm.ensure((size_t)V * 4 + 16));
    OLV_TRY(ws.sr_newid.ensure((size_t)V * 4 + 16));
    OLV_TRY(ws.sr_rowptr.ensure(((size_t)V + 1) * 4 + 16));
    OLV_TRY(ws.sr_colptr.ensure(((size_t)V + 1) * 4 + 16));
    OLV_TRY(ws.sr_col.ensure(E * 4 + 16));
    OLV_TRY(ws.sr_w.ensure(E * 4 + 16));
    OLV_TRY(ws.sr_rowidx.ensure(E * 4 + 16));
    OLV_TRY(ws.sr_cw.ensure(E * 4 + 16));
    OLV_TRY(ws.sr_dist.ensure((size_t)V * 4 + 16));
    OLV_CUDA(cudaMemcpyAsync(ws.sr_perm.p, perm.data(), (size_t)V * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(ws.sr_newid.p, newid.data(), (size_t)V * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(ws.sr_rowptr.p, nrp.data(), ((size_t)V + 1) * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(ws.sr_colptr.p, ncp.data(), ((size_t)V + 1) * 4, cudaMemcpyHostToDevice, s));
    if (E) {
        k_sssp_relabel<<<g->num_sms * 16, kBlock, 0, s>>>(
            g->rowptr.as<uint32_t>(), g->col.as<uint32_t>(), g->w.as<uint32_t>(),
            ws.sr_perm.as<uint32_t>(), ws.sr_newid.as<uint32_t>(), ws.sr_rowptr.as<uint32_t>(), V,
            ws.sr_col.as<uint32_t>(), ws.sr_w.as<uint32_t>());
        k_sssp_relabel<<<g->num_sms * 16, kBlock, 0, s>>>(
            g->colptr.as<uint32_t>(), g->rowidx.as<uint32_t>(), g->csc_w.as<uint32_t>(),
            ws.sr_perm.as<uint32_t>(), ws.sr_newid.as<uint32_t>(), ws.sr_colptr.as<uint32_t>(), V,
            ws.sr_rowidx.as<uint32_t>(), ws.sr_cw.as<uint32_t>());
        OLV_CUDA(cudaGetLastError());
    }
    OLV_CUDA(cudaStreamSynchronize(s));   // the host vectors die here
    ws.sr_built = 1;
    return OLV_OK;
}

// The graph SSSP runs on: renumbered (sssp_relabel) or the handle's own.
struct SsspCsr {
    const uint32_t *rowptr, *col, *w, *colptr, *rowidx, *cw, *newid;
    uint32_t *dist;   // internal distances (renumbered run), else null
};
static SsspCsr sssp_csr(olv_graph *g) {
    Workspace &ws = g->ws;
    if (g->tune.sssp_relabel && ws.sr_built)
        return SsspCsr{ws.sr_rowptr.as<uint32_t>(), ws.sr_col.as<uint32_t>(),
                       ws.sr_w.as<uint32_t>(),      ws.sr_colptr.as<uint32_t>(),
                       ws.sr_rowidx.as<uint32_t>(), ws.sr_cw.as<uint32_t>(),
                       ws.sr_newid.as<uint32_t>(),  ws.sr_dist.as<uint32_t>()};
    return SsspCsr{g->rowptr.as<uint32_t>(), g->col.as<uint32_t>(),    g->w.as<uint32_t>(),
                   g->colptr.as<uint32_t>(), g->rowidx.as<uint32_t>(), g->csc_w.as<uint32_t>(),
                   nullptr,                  nullptr};
}

// Rows split light | heavy for the current delta (built once per delta and
// numbering).
static int sssp_partition(olv_graph *g) {
    Workspace &ws = g->ws;
    const uint32_t delta = sssp_delta(g);
    if (g->tune.sssp_relabel) OLV_TRY(sssp_relabel(g));
    const int relabel = g->tune.sssp_relabel ? 1 : 0;
    if (ws.sssp_delta_built == delta && ws.sssp_part_relabel == relabel && ws.rowmid.p)
        return OLV_OK;
    const SsspCsr R = sssp_csr(g);
    OLV_TRY(ws.sssp_cw.ensure(g->E * 8 + 16));
    OLV_TRY(ws.rowmid.ensure((size_t)g->V * 4 + 16));
    OLV_TRY(ws.sssp_lr.ensure((size_t)g->V * 8 + 16));
    OLV_TRY(ws.sssp_hr.ensure((size_t)g->V * 8 + 16));
    OLV_TRY(ws.hdin.ensure((size_t)g->V * 8 + 16));
    k_partition_rows<<<g->num_sms * 16, kBlock, 0, g->stream>>>(
        R.rowptr, R.col, R.w, g->V, delta, ws.sssp_cw.as<uint2>(), ws.rowmid.as<uint32_t>(),
        ws.sssp_lr.as<uint2>(), ws.sssp_hr.as<uint2>());
    k_heavy_in_degrees<<<g->num_sms * 8, kBlock, 0, g->stream>>>(
        R.rowptr, ws.rowmid.as<uint32_t>(), R.colptr, g->V, ws.hdin.as<uint2>());
    if (R.cw && R.rowidx) {   // in-edges as (source, weight) pairs for the pull
        OLV_TRY(ws.sssp_crw.ensure(g->E * 8 + 16));
        k_pack_pairs<<<g->num_sms * 8, kBlock, 0, g->stream>>>(R.rowidx, R.cw, g->E,
                                                              ws.sssp_crw.as<uint2>());
    }
    OLV_CUDA(cudaGetLastError());
    ws.sssp_delta_built = delta;
    ws.sssp_part_relabel = relabel;
    return OLV_OK;
}

template <class Sink>
static int sssp_superstep(olv_graph *g, Sink &&sink, cudaGraphConditionalHandle h,
                          int use_cond) {
    Workspace &ws = g->ws;
    TravCtl *ctl = ws.ctl.as<TravCtl>();
    const SsspCsr R = sssp_csr(g);
    AdvanceArgs a;   // light edges: [rowptr[u], rowmid[u]) = sssp_lr[u]
    a.rng = ws.sssp_lr.as<uint2>();
    a.cw = ws.sssp_cw.as<uint2>();
    a.ctl = ctl;
    a.q0 = ws.q0.as<uint32_t>();
    a.q1 = ws.q1.as<uint32_t>();
    a.far0 = ws.far0.as<uint32_t>();
    a.far1 = ws.far1.as<uint32_t>();
    a.pieces = ws.pieces.as<uint2>();
    a.hub_degree = g->tune.sssp_hub_degree;
    a.piece = g->tune.sssp_piece;
    a.want_mode = kModeRelax;
    SsspOp op = {};
    const size_t words = mark_words(g->V);
    uint32_t *mk = ws.mark.as<uint32_t>();
    op.nmark0 = mk;
    op.nmark1 = mk + words;
    op.fmark0 = mk + 2 * words;
    op.fmark1 = mk + 3 * words;
    FarMarks fm;
    fm.m0 = op.fmark0;
    fm.m1 = op.fmark1;
    uint32_t *q0 = a.q0, *q1 = a.q1, *far0 = a.far0, *far1 = a.far1;
    // a correct run needs far fewer supersteps; the bound only stops a runaway loop
    uint32_t max_steps = (uint32_t)(3ULL * g->V + 1000 > 0xfffffff0ULL ? 0xfffffff0ULL
                                                                    : 3ULL * g->V + 1000);
    // the relax kernel for the tuned sources per thread (1, 2, 4 or 8)
    const uint32_t spt = g->tune.sssp_spt;
    const void *chunks = spt == 8   ? (const void *)k_advance_chunks<SsspOp, 8>
                         : spt == 4 ? (const void *)k_advance_chunks<SsspOp, 4>
                         : spt == 2 ? (const void *)k_advance_chunks<SsspOp, 2>
                                    : (const void *)k_advance_chunks<SsspOp, 1>;
    int nb = 0;   // the relax kernel's own residency (it holds more registers than BFS's)
    OLV_TRY(resident_blocks(g, chunks, &nb));
    uint32_t V = g->V;
    a.rng2 = ws.sssp_hr.as<uint2>();   // heavy edges: [rowmid[u], rowptr[u+1])
    a.want_mode2 = kModeHeavy;
    a.rbeg3 = R.rowptr;                // every edge: [rowptr[u], rowptr[u+1])
    a.rend3 = R.rowptr + 1;
    a.want_mode3 = kModeRelaxAll;
    SsspAux x;
    x.colptr = R.colptr;
    x.crw = ws.sssp_crw.as<uint2>();
    x.vpull = R.newid ? ws.sr_vnz : V;
    // renumbered: rows past the long-in-degree prefix (rounded up to whole
    // chunks) are short and go a thread per vertex; otherwise all by chunks
    const uint32_t ps = g->tune.sssp_pull_split;   // 0 or the short-row bound 4, 8, 16, 32
    const uint32_t vlong = ws.sr_vlong[ps >= 32 ? 3 : ps >= 16 ? 2 : ps >= 8 ? 1 : 0];
    x.vsplit = R.newid && ps ? (uint32_t)std::min<uint64_t>(
                                   ((uint64_t)vlong + kPullChunk - 1) / kPullChunk * kPullChunk,
                                   x.vpull)
                             : x.vpull;
    x.E = g->E;
    x.hdin = ws.hdin.as<uint2>();
    x.blist = ws.blist.as<uint32_t>();
    x.cmark = mk + 4 * words;
    x.mark_words = (uint32_t)words;
    x.bl_cap = V;
    x.pull = g->tune.sssp_pull && x.crw != nullptr;
    void *a_aux[] = {&V, &ctl, &q0, &q1, &far0, &far1, &fm, &x};
    // the dense passes on 2 CTAs per SM: measured faster than 3 or 4 on
    // RMAT-24 (1.68-1.69 ms against 1.79-1.81 at 4), the idle launches of the
    // relax supersteps cost less and the pull's chunks stay as balanced
    const int nba = 2 * g->num_sms;
    OLV_TRY(sink((const void *)k_sssp_aux, dim3(nba), dim3(kBlock), a_aux));
    uint32_t bl_cap = x.bl_cap;
    // the end step runs in the pieces kernel's last CTA, or as its own launch
    op.end_h = h;
    op.end_fused = g->tune.sssp_fuse_end;
    op.end_use_cond = use_cond;
    op.end_max_steps = max_steps;
    op.end_bl_cap = bl_cap;
    void *a_adv[] = {&a, &op};
    OLV_TRY(sink(chunks, dim3(nb), dim3(kBlock), a_adv));
    OLV_TRY(sink((const void *)k_advance_pieces<SsspOp>, dim3(nb), dim3(kBlock), a_adv));
    if (!op.end_fused) {
        void *a_end[] = {&ctl, &h, &use_cond, &max_steps, &bl_cap};
        OLV_TRY(sink((const void *)k_sssp_end, dim3(1), dim3(1), a_end));
    }
    return OLV_OK;
}

static int sssp_graph(olv_graph *g) {
    if (g->sssp_graph && g->sssp_graph->ready) return OLV_OK;
    if (!g->sssp_graph) g->sssp_graph = new WhileGraph();
    WhileGraph &wg = *g->sssp_graph;
    OLV_TRY(wg.begin());
    auto sink = [&](const void *f, dim3 gr, dim3 bl, void **args) { return wg.add(f, gr, bl, args); };
    OLV_TRY(sssp_superstep(g, sink, wg.handle, 1));
    return wg.finish();
}

int sssp_workspace(olv_graph *g) {
    OLV_TRY(traversal_workspace(g, true));
    const size_t V = g->V;
    OLV_TRY(g->ws.far0.ensure(V * 4 + 16));
    OLV_TRY(g->ws.far1.ensure(V * 4 + 16));
    OLV_TRY(g->ws.blist.ensure(V * 4 + 16));
    OLV_TRY(g->ws.mark.ensure(kMarks * mark_words(V) * 4));
    return OLV_OK;
}

// red (device, [2], zeroed; or null): reached out-edges and vertices, summed
// by the final pass when the run is renumbered; *red_done says whether it was.
int run_sssp_device(olv_graph *g, uint32_t src, uint32_t *dist_dev, unsigned long long *red,
                    bool *red_done) {
    *red_done = false;
    OLV_TRY(sssp_partition(g));
    cudaStream_t s = g->stream;
    TravCtl *ctl = g->ws.ctl.as<TravCtl>();
    const SsspCsr R = sssp_csr(g);
    uint32_t *dist = R.dist ? R.dist : dist_dev;   // renumbered run: internal distances
    OLV_CUDA(cudaMemsetAsync(g->ws.mark.p, 0, kMarks * mark_words(g->V) * 4, s));
    k_fill_i32<<<g->num_sms * 8, kBlock, 0, s>>>((int32_t *)dist, g->V, kInf);
    k_sssp_init<<<1, 1, 0, s>>>(ctl, dist, g->ws.q0.as<uint32_t>(), src, sssp_delta(g),
                                g->tune.sssp_sub, g->tune.sssp_sub_buckets,
                                g->tune.sssp_tail_delta, g->tune.sssp_route,
                                g->tune.sssp_pull_direct && g->tune.sssp_pull && g->ws.sssp_crw.p
                                    ? std::max<uint32_t>(1u, g->V / 16) : 0u,
                                R.newid);
    OLV_CUDA(cudaGetLastError());
    auto finish = [&]() -> int {
        if (R.dist) {
            k_sssp_unrelabel<<<g->num_sms * 8, kBlock, 0, s>>>(R.dist, R.newid, g->V, dist_dev,
                                                              g->rowptr.as<uint32_t>(), red);
            OLV_CUDA(cudaGetLastError());
            *red_done = red != nullptr;
        }
        return OLV_OK;
    };
    if (g->tune.use_graphs) {
        if (sssp_graph(g) == OLV_OK) {
            OLV_TRY(g->sssp_graph->launch(s));
            return finish();
        }
        g->tune.use_graphs = 0;
    }
    auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
        OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
        return OLV_OK;
    };
    for (;;) {
        for (int i = 0; i < g->tune.levels_per_sync; i++) OLV_TRY(sssp_superstep(g, launch, 0, 0));
        OLV_CUDA(cudaMemcpyAsync(g->host_ctl, ctl, sizeof(TravCtl), cudaMemcpyDeviceToHost, s));
        OLV_CUDA(cudaStreamSynchronize(s));
        if (g->host_ctl->done) break;
    }
    return finish();
}

}  // namespace olv

using namespace olv;

extern "C" int olv_sssp(olv_graph *g, uint32_t src, uint32_t *dist_out, olv_stats *st) {
    OLV_CHECK_ARG(g && dist_out, "olv_sssp: null pointer");
    OLV_CHECK_ARG(src < g->V, "olv_sssp: source %u out of range (V=%u)", src, g->V);
    OLV_CHECK_ARG(g->weight_type == OLV_W_U32, "olv_sssp: graph has no uint32 weights");
    OLV_TRY(sssp_workspace(g));
    const bool dev_out = is_device_ptr(dist_out);
    if (!dev_out) OLV_TRY(g->ws.level.ensure((size_t)g->V * 4 + 16));
    uint32_t *dist = dev_out ? dist_out : g->ws.level.as<uint32_t>();
    cudaStream_t s = g->stream;
    unsigned long long *red_dev = nullptr;
    if (st) {
        OLV_TRY(g->ws.tmp.ensure(16));
        OLV_CUDA(cudaMemsetAsync(g->ws.tmp.p, 0, 16, s));
        red_dev = g->ws.tmp.as<unsigned long long>();
    }
    bool red_done = false;
    OLV_CUDA(cudaEventRecord(g->ev0, s));
    OLV_TRY(run_sssp_device(g, src, dist, red_dev, &red_done));
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    OLV_CUDA(cudaMemcpyAsync(g->host_ctl, g->ws.ctl.p, sizeof(TravCtl), cudaMemcpyDeviceToHost, s));
    unsigned long long red[2] = {0, 0};
    if (st) {
        if (!red_done)
            k_reached_edges<<<g->num_sms * 4, kBlock, 0, s>>>(g->rowptr.as<uint32_t>(), dist, g->V,
                                                             red_dev);
        OLV_CUDA(cudaMemcpyAsync(red, red_dev, 16, cudaMemcpyDeviceToHost, s));
    }
    if (!dev_out)
        OLV_CUDA(cudaMemcpyAsync(dist_out, dist, (size_t)g->V * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    const TravCtl &h = *g->host_ctl;
    if (h.err) {
        set_error("olv_sssp: device-side check failed (code %u)", h.err);
        return OLV_ERR_STATE;
    }
    if (st) {
        float ms = 0;
        OLV_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        st->iterations = h.steps;
        st->pull_steps = 0;
        st->vertices_reached = red[1];
        st->edges_traversed = red[0];
        st->edges_relaxed = h.edges_relaxed;
        st->residual = 0;
        st->device_ms = ms;
    }
    return OLV_OK;
}
