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
#include "olv_advance.cuh"
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"

namespace olv {

int traversal_workspace(olv_graph *g, bool pieces);
__global__ void k_fill_i32(int32_t *__restrict__ a, uint32_t n, int32_t x);

constexpr uint32_t kModeRelax = 0;
constexpr uint32_t kModeSplit = 2;
constexpr uint32_t kModeHeavy = 3;
constexpr uint32_t kDefaultDelta = 64;

// Stable partition of every row into light (w <= delta) then heavy edges; one
// warp per row, two passes (count, then write in order).
__global__ void k_partition_rows(const uint32_t *__restrict__ rowptr,
                                 const uint32_t *__restrict__ col, const uint32_t *__restrict__ w,
                                 uint32_t V, uint32_t delta, uint32_t *__restrict__ pcol,
                                 uint32_t *__restrict__ pw, uint32_t *__restrict__ rowmid) {
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
            if (light) {
                pcol[lo + __popc(ml & lt)] = ci;
                pw[lo + __popc(ml & lt)] = wi;
            } else if (ok) {
                pcol[hi + __popc(mh & lt)] = ci;
                pw[hi + __popc(mh & lt)] = wi;
            }
            lo += __popc(ml);
            hi += __popc(mh);
        }
        if (lane == 0) rowmid[u] = b + nl;
    }
}

#ifndef OLV_SSSP_MINB
#define OLV_SSSP_MINB 4   // 4: <= 64 registers
#endif
struct SsspOp {
    static constexpr int kMinBlocks = OLV_SSSP_MINB;   // CTAs per SM the advance must fit
    using SV = uint32_t;
    static constexpr bool kHasFar = true;
    const uint32_t *w;
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
    __device__ __forceinline__ Pre prepare(uint32_t du, uint32_t e, uint32_t v) const {
        uint32_t nd = du + __ldcs(&w[e]);   // streamed once: evict first
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
    // the input vertex was queued (and marked) by the previous superstep
    __device__ __forceinline__ void on_input(uint32_t u) const {
        atomicAnd(&nprev[u >> 5], ~(1u << (u & 31)));
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
                            uint32_t delta) {
    TravCtl t = {};
    t.qsize[0] = 1;
    t.vdata = dist;
    t.threshold = delta;
    t.delta = delta;
    t.epoch = 1;
    t.far_min = 0xffffffffu;
    t.heavy_done = 0;
    t.bucket_lo = 0;
    *c = t;
    dist[src] = 0;
    q0[0] = src;
    sssp_begin(c);
}

// Choose the next superstep's mode (relax light edges, relax a settled
// bucket's heavy edges, or split the far pile) and reset its counters.
__device__ void sssp_begin(TravCtl *c) {
    if (c->done) return;
    if (c->qsize[c->cur] > 0) {
        c->mode = kModeRelax;
        c->qsize[c->cur ^ 1] = 0;
        c->npieces = 0;
        return;
    }
    if (!c->heavy_done) {   // bucket settled: collect it and relax its heavy edges
        c->mode = kModeHeavy;
        c->qsize[c->cur] = 0;
        c->qsize[c->cur ^ 1] = 0;
        c->npieces = 0;
        return;
    }
    if (c->far_size[c->far_cur] == 0) {
        c->done = 1;
        return;
    }
    // next bucket starts at max(threshold, smallest far distance)
    c->mode = kModeSplit;
    c->split_lo = c->threshold;   // far entries below it were settled already
    c->bucket_lo = c->threshold;
    uint32_t lo = c->threshold > c->far_min ? c->threshold : c->far_min;
    uint64_t t = (uint64_t)lo + c->delta;
    c->threshold = t > (uint64_t)kInf ? (uint32_t)kInf : (uint32_t)t;
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
// [bucket_lo, threshold) become the input queue.  Four vertices per thread.
__device__ void sssp_collect(uint32_t V, TravCtl *c, uint32_t *q0, uint32_t *q1,
                             WarpStage st) {
    const uint32_t *dist = static_cast<const uint32_t *>(c->vdata);
    const uint32_t lo = c->bucket_lo, hi = c->threshold;
    uint32_t *q = c->cur ? q1 : q0;
    uint32_t *qsize = &c->qsize[c->cur];
    const bool vec = ((uintptr_t)dist & 15) == 0;
    const uint64_t nquad = ((uint64_t)V + 3) / 4;
    for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < nquad;
         base += (uint64_t)gridDim.x * kBlock) {
        const uint64_t v0 = (base + threadIdx.x) * 4;
        uint32_t d[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
        if (vec && v0 + 3 < V) {
            const uint4 x = __ldcg(reinterpret_cast<const uint4 *>(dist + v0));
            d[0] = x.x;
            d[1] = x.y;
            d[2] = x.z;
            d[3] = x.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (v0 + j < V) d[j] = __ldcg(dist + v0 + j);
        }
        int act[4];
        uint32_t vv[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            act[j] = d[j] >= lo && d[j] < hi;   // vertices >= V hold 0xffffffff
            vv[j] = (uint32_t)(v0 + j);
        }
        st.reserve(32 * 4, q, qsize);
        stage_push_n<4>(act, vv, 1, st.buf, st.n, st.lim, kWarpStage, q, qsize);
    }
    warp_stage_flush(st.buf, st.n, st.lim, q, qsize);
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

__global__ void k_sssp_end(TravCtl *c, cudaGraphConditionalHandle h, int use_cond,
                           uint32_t max_steps) {
    if (!c->done) {
        if (c->mode == kModeRelax) {
            c->cur ^= 1;
        } else if (c->mode == kModeHeavy) {
            c->qsize[c->cur] = 0;
            c->heavy_done = 1;
        } else {
            c->far_cur ^= 1;
            c->epoch++;
            c->heavy_done = 0;
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

// The superstep's dense pass: collect the settled bucket (heavy mode) or split
// the far pile (split mode); nothing in relax mode.
__global__ void __launch_bounds__(kBlock)
k_sssp_aux(uint32_t V, TravCtl *c, uint32_t *q0, uint32_t *q1, uint32_t *far0, uint32_t *far1,
           FarMarks fm) {
    if (c->done) return;
    const uint32_t mode = c->mode;
    if (mode != kModeHeavy && mode != kModeSplit) return;
    __shared__ uint32_t s_a[kBlock / 32][kWarpStage], s_b[kBlock / 32][kWarpStage];
    __shared__ uint32_t s_an[kBlock / 32], s_alim[kBlock / 32];
    __shared__ uint32_t s_bn[kBlock / 32], s_blim[kBlock / 32];
    const uint32_t wl = threadIdx.x >> 5;
    WarpStage sa{s_a[wl], &s_an[wl], &s_alim[wl]};
    WarpStage sb{s_b[wl], &s_bn[wl], &s_blim[wl]};
    sa.init();
    sb.init();
    if (mode == kModeHeavy)
        sssp_collect(V, c, q0, q1, sa);
    else
        sssp_split(c, q0, q1, far0, far1, fm, sa, sb);
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

static uint32_t sssp_delta(olv_graph *g) {
    if (g->tune.sssp_delta) return g->tune.sssp_delta;
    return kDefaultDelta;
}

// Rows split light | heavy for the current delta (built once per delta).
static int sssp_partition(olv_graph *g) {
    Workspace &ws = g->ws;
    const uint32_t delta = sssp_delta(g);
    if (ws.sssp_delta_built == delta && ws.rowmid.p) return OLV_OK;
    OLV_TRY(ws.sssp_col.ensure(g->E * 4 + 16));
    OLV_TRY(ws.sssp_w.ensure(g->E * 4 + 16));
    OLV_TRY(ws.rowmid.ensure((size_t)g->V * 4 + 16));
    k_partition_rows<<<g->num_sms * 16, kBlock, 0, g->stream>>>(
        g->rowptr.as<uint32_t>(), g->col.as<uint32_t>(), g->w.as<uint32_t>(), g->V, delta,
        ws.sssp_col.as<uint32_t>(), ws.sssp_w.as<uint32_t>(), ws.rowmid.as<uint32_t>());
    OLV_CUDA(cudaGetLastError());
    ws.sssp_delta_built = delta;
    return OLV_OK;
}

template <class Sink>
static int sssp_superstep(olv_graph *g, Sink &&sink, cudaGraphConditionalHandle h,
                          int use_cond) {
    Workspace &ws = g->ws;
    TravCtl *ctl = ws.ctl.as<TravCtl>();
    AdvanceArgs a;   // light edges: [rowptr[u], rowmid[u])
    a.rbeg = g->rowptr.as<uint32_t>();
    a.rend = ws.rowmid.as<uint32_t>();
    a.col = ws.sssp_col.as<uint32_t>();
    a.ctl = ctl;
    a.q0 = ws.q0.as<uint32_t>();
    a.q1 = ws.q1.as<uint32_t>();
    a.far0 = ws.far0.as<uint32_t>();
    a.far1 = ws.far1.as<uint32_t>();
    a.pieces = ws.pieces.as<uint2>();
    a.hub_degree = g->tune.hub_degree;
    a.piece = g->tune.piece;
    a.want_mode = kModeRelax;
    AdvanceArgs ah = a;   // heavy edges: [rowmid[u], rowptr[u+1])
    ah.rbeg = ws.rowmid.as<uint32_t>();
    ah.rend = g->rowptr.as<uint32_t>() + 1;
    SsspOp op = {};
    op.w = ws.sssp_w.as<uint32_t>();
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
    int nb = 0;   // the relax kernel's own residency (it holds more registers than BFS's)
    OLV_TRY(resident_blocks(g, (const void *)k_advance_chunks<SsspOp>, &nb));
    uint32_t V = g->V;
    a.rbeg2 = ah.rbeg;
    a.rend2 = ah.rend;
    a.want_mode2 = kModeHeavy;
    void *a_aux[] = {&V, &ctl, &q0, &q1, &far0, &far1, &fm};
    OLV_TRY(sink((const void *)k_sssp_aux, dim3(nb), dim3(kBlock), a_aux));
    void *a_adv[] = {&a, &op};
    OLV_TRY(sink((const void *)k_advance_chunks<SsspOp>, dim3(nb), dim3(kBlock), a_adv));
    OLV_TRY(sink((const void *)k_advance_pieces<SsspOp>, dim3(nb), dim3(kBlock), a_adv));
    void *a_end[] = {&ctl, &h, &use_cond, &max_steps};
    OLV_TRY(sink((const void *)k_sssp_end, dim3(1), dim3(1), a_end));
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
    OLV_TRY(g->ws.mark.ensure(4 * mark_words(V) * 4));
    return OLV_OK;
}

int run_sssp_device(olv_graph *g, uint32_t src, uint32_t *dist_dev) {
    OLV_TRY(sssp_partition(g));
    cudaStream_t s = g->stream;
    TravCtl *ctl = g->ws.ctl.as<TravCtl>();
    OLV_CUDA(cudaMemsetAsync(g->ws.mark.p, 0, 4 * mark_words(g->V) * 4, s));
    k_fill_i32<<<g->num_sms * 8, kBlock, 0, s>>>((int32_t *)dist_dev, g->V, kInf);
    k_sssp_init<<<1, 1, 0, s>>>(ctl, dist_dev, g->ws.q0.as<uint32_t>(), src, sssp_delta(g));
    OLV_CUDA(cudaGetLastError());
    if (g->tune.use_graphs) {
        if (sssp_graph(g) == OLV_OK) return g->sssp_graph->launch(s);
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
    return OLV_OK;
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
    OLV_CUDA(cudaEventRecord(g->ev0, s));
    OLV_TRY(run_sssp_device(g, src, dist));
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    OLV_CUDA(cudaMemcpyAsync(g->host_ctl, g->ws.ctl.p, sizeof(TravCtl), cudaMemcpyDeviceToHost, s));
    unsigned long long red[2] = {0, 0};
    if (st) {
        OLV_TRY(g->ws.tmp.ensure(16));
        OLV_CUDA(cudaMemsetAsync(g->ws.tmp.p, 0, 16, s));
        k_reached_edges<<<g->num_sms * 4, kBlock, 0, s>>>(g->rowptr.as<uint32_t>(), dist, g->V,
                                                         g->ws.tmp.as<unsigned long long>());
        OLV_CUDA(cudaMemcpyAsync(red, g->ws.tmp.p, 16, cudaMemcpyDeviceToHost, s));
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
