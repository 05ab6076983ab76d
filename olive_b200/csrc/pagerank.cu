// PageRank: deterministic FP32 pull over the reverse graph.
//
// Result contract: PageRank.cu:89-147 / testPageRank.cu:41-115 -- ranks start
// at 1/N; each iteration r'[v] = (1-alpha)/N + alpha * sum_{u->v} r[u]/outdeg(u)
// (+ alpha * d/N with d the dangling mass when it is redistributed); stop when
// the L1 change sum|r' - r| < tol or after max_it iterations.
//
// The reference pushes rank/outdeg along out-edges with an FP64 CAS atomicAdd
// (PageRank.cu:51-61, common.h:141-150), refills the V accumulators on the host
// every iteration (oliver.h:127) and copies all vertex values back to sum the
// residual on the host (oliver.h:176-183).  Here:
//   * each iteration is one pull kernel over the in-edges (CSC).  Vertices are
//     cut into row blocks of at most kNnz in-edges; a CTA stages its block's
//     contributions in shared memory and each thread sums whole rows in CSC
//     order with compensated (two-sum) FP32 arithmetic, so results do not
//     depend on scheduling and carry ~1 rounding per vertex;  a row longer
//     than kNnz gets a CTA of its own and a fixed-shape tree;
//   * the same kernel writes the next iteration's contributions r/outdeg and
//     per-CTA FP64 partial sums of |r' - r| and of the dangling mass;
//   * a one-CTA kernel folds the partials in a fixed order (FP64), decides
//     convergence on the device and sets the loop condition of the CUDA graph
//     that runs all iterations.
#include <algorithm>
#include <vector>

#include "olv_advance.cuh"
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"

namespace olv {

constexpr uint32_t kNnz = 2048;      // in-edges staged per row block
constexpr uint32_t kRows = 2048;     // rows per row block at most
constexpr uint32_t kSeg = 4096;      // in-edges per segment of a long row
constexpr int kRedThreads = 1024;
constexpr int kGather = kNnz / kBlock;

struct PrCtl {
    double base;        // (1-alpha)/N + alpha*d/N for the running iteration
    double residual;    // L1 change of the last completed iteration
    double dangling;
    uint32_t iter;      // completed iterations
    uint32_t done;
    uint32_t max_it;
    uint32_t leak;
    double tol;
    double alpha;
    double inv_n;
};

// (s, c) <- s + x with the rounding error of the addition accumulated in c.
__device__ __forceinline__ void two_sum_acc(float &s, float &c, float x) {
    const float t = s + x;
    const float bp = t - s;
    c += (s - (t - bp)) + (x - bp);
    s = t;
}

__device__ __forceinline__ void pair_add(float &s, float &c, float s2, float c2) {
    two_sum_acc(s, c, s2);
    c += c2;
}

// r' = alpha * (s + c) + base, with alpha split into hi + lo FP32 parts.
__device__ __forceinline__ float pr_update(float s, float c, float a_hi, float a_lo, float base) {
    const float t = fmaf(a_lo, s, fmaf(a_hi, c, base));
    return fmaf(a_hi, s, t);
}

__global__ void __launch_bounds__(kBlock)
k_pr_pull(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowidx,
          const uint32_t *__restrict__ blocks, const uint32_t *__restrict__ outdeg,
          const float *c0, const float *c1, float *__restrict__ rank, PrCtl *ctl,
          double *__restrict__ partials, float a_hi, float a_lo,
          const uint32_t *__restrict__ segbase, const float2 *__restrict__ segs) {
    if (ctl->done) return;
    const float *__restrict__ cin = (ctl->iter & 1) ? c1 : c0;
    float *__restrict__ cout = (float *)((ctl->iter & 1) ? c0 : c1);
    const float base = (float)ctl->base;
    const uint32_t r0 = blocks[blockIdx.x], r1 = blocks[blockIdx.x + 1];
    const uint32_t e0 = colptr[r0], e1 = colptr[r1];
    __shared__ float s_val[kNnz];
    __shared__ double s_dred[2][kBlock / 32];
    double res = 0.0, dang = 0.0;

    auto finish_row = [&](uint32_t v, float s, float c) {
        const float nr = pr_update(s, c, a_hi, a_lo, base);
        const float old = rank[v];
        rank[v] = nr;
        res += fabs((double)nr - (double)old);
        const uint32_t d = outdeg[v];
        if (d) {
            cout[v] = __fdiv_rn(nr, (float)d);
        } else {
            cout[v] = 0.0f;
            dang += (double)nr;
        }
    };

    if (e1 - e0 <= kNnz) {
        const uint32_t n = e1 - e0;
        uint32_t idx[kGather];
#pragma unroll
        for (int j = 0; j < kGather; j++) {
            const uint32_t i = threadIdx.x + j * kBlock;
            idx[j] = i < n ? __ldg(&rowidx[e0 + i]) : 0u;
        }
#pragma unroll
        for (int j = 0; j < kGather; j++) {
            const uint32_t i = threadIdx.x + j * kBlock;
            if (i < n) s_val[i] = __ldg(&cin[idx[j]]);
        }
        __syncthreads();
        for (uint32_t v = r0 + threadIdx.x; v < r1; v += kBlock) {
            const uint32_t b = colptr[v] - e0, e = colptr[v + 1] - e0;
            float s = 0.0f, c = 0.0f;
            for (uint32_t i = b; i < e; i++) two_sum_acc(s, c, s_val[i]);
            finish_row(v, s, c);
        }
    } else if (threadIdx.x == 0) {
        // one long row: its segments were summed by k_pr_segments; fold in order
        const uint32_t first = segbase[blockIdx.x];
        const uint32_t nseg = (e1 - e0 + kSeg - 1) / kSeg;
        float s = 0.0f, c = 0.0f;
        for (uint32_t k = 0; k < nseg; k++) {
            const float2 p = segs[first + k];
            pair_add(s, c, p.x, p.y);
        }
        finish_row(r0, s, c);
    }
    // fixed-order CTA reduction of the FP64 partials
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        res += __shfl_down_sync(0xffffffffu, res, o);
        dang += __shfl_down_sync(0xffffffffu, dang, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_dred[0][threadIdx.x >> 5] = res;
        s_dred[1][threadIdx.x >> 5] = dang;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int i = 0; i < kBlock / 32; i++) {
            a += s_dred[0][i];
            b += s_dred[1][i];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

// Compensated sums of the kSeg-edge segments of long rows: thread t sums
// elements t, t+kBlock, ... of its segment, then a fixed-shape tree.
__global__ void __launch_bounds__(kBlock)
k_pr_segments(const uint32_t *__restrict__ rowidx, const uint2 *__restrict__ seg_range,
              const float *c0, const float *c1, const PrCtl *ctl, float2 *__restrict__ segs) {
    if (ctl->done) return;
    const float *__restrict__ cin = (ctl->iter & 1) ? c1 : c0;
    const uint2 r = seg_range[blockIdx.x];
    __shared__ float s_red[2][kBlock];
    float s = 0.0f, c = 0.0f;
    constexpr int U = kSeg / kBlock;
    uint32_t idx[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
        const uint32_t i = r.x + threadIdx.x + j * kBlock;
        idx[j] = i < r.y ? __ldg(&rowidx[i]) : 0xffffffffu;
    }
    float x[U];
#pragma unroll
    for (int j = 0; j < U; j++) x[j] = idx[j] != 0xffffffffu ? __ldg(&cin[idx[j]]) : 0.0f;
#pragma unroll
    for (int j = 0; j < U; j++) two_sum_acc(s, c, x[j]);
    s_red[0][threadIdx.x] = s;
    s_red[1][threadIdx.x] = c;
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < (uint32_t)w) {
            float a = s_red[0][threadIdx.x], ac = s_red[1][threadIdx.x];
            pair_add(a, ac, s_red[0][threadIdx.x + w], s_red[1][threadIdx.x + w]);
            s_red[0][threadIdx.x] = a;
            s_red[1][threadIdx.x] = ac;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) segs[blockIdx.x] = make_float2(s_red[0][0], s_red[1][0]);
}

// Fold the per-CTA partials (fixed order), publish residual and the next
// iteration's constant term, decide convergence.
__global__ void __launch_bounds__(kRedThreads)
k_pr_reduce(PrCtl *ctl, const double *__restrict__ partials, uint32_t nparts,
            cudaGraphConditionalHandle h, int use_cond) {
    __shared__ double s[2][kRedThreads];
    if (ctl->done) {
        if (use_cond && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
        return;
    }
    double a = 0, b = 0;
    for (uint32_t i = threadIdx.x; i < nparts; i += kRedThreads) {
        a += partials[2 * i];
        b += partials[2 * i + 1];
    }
    s[0][threadIdx.x] = a;
    s[1][threadIdx.x] = b;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < (uint32_t)w) {
            s[0][threadIdx.x] += s[0][threadIdx.x + w];
            s[1][threadIdx.x] += s[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double res = s[0][0], dang = s[1][0];
        ctl->residual = res;
        ctl->dangling = dang;
        ctl->iter++;
        ctl->base = (1.0 - ctl->alpha) * ctl->inv_n +
                    (ctl->leak ? 0.0 : ctl->alpha * dang * ctl->inv_n);
        if (res < ctl->tol || ctl->iter >= ctl->max_it) ctl->done = 1;
        if (use_cond) cudaGraphSetConditional(h, ctl->done ? 0u : 1u);
    }
}

// r = 1/N, contributions r/outdeg, count of dangling vertices (exact integer
// count, so the first constant term does not depend on atomic ordering).
__global__ void k_pr_init(const uint32_t *__restrict__ outdeg, uint32_t V, float *rank, float *c0,
                          unsigned long long *ndang) {
    const float r = __fdiv_rn(1.0f, (float)V);
    unsigned long long nd = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        rank[v] = r;
        const uint32_t d = outdeg[v];
        c0[v] = d ? __fdiv_rn(r, (float)d) : 0.0f;
        nd += d == 0;
    }
    warp_add64(nd, ndang);
}

__global__ void k_pr_ctl_init(PrCtl *ctl, const unsigned long long *ndang, uint32_t V,
                              double alpha, uint32_t max_it, double tol, uint32_t leak) {
    PrCtl c = {};
    c.alpha = alpha;
    c.inv_n = 1.0 / (double)V;
    c.tol = tol;
    c.max_it = max_it;
    c.leak = leak;
    const double dang = (double)(*ndang) * (double)__fdiv_rn(1.0f, (float)V);
    c.dangling = dang;
    c.base = (1.0 - alpha) * c.inv_n + (leak ? 0.0 : alpha * dang * c.inv_n);
    c.residual = 0;
    c.done = max_it == 0;
    *ctl = c;
}

__global__ void k_outdeg(const uint32_t *__restrict__ rowptr, uint32_t V, uint32_t *d) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x)
        d[v] = rowptr[v + 1] - rowptr[v];
}

// ------------------------------------------------------------------ host --
struct PrPlan {
    DevBuf blocks, outdeg, contrib, partials, ctl, dang, segbase, seg_range, segs;
    uint32_t nblocks = 0;
    uint32_t nsegs = 0;
    float a_hi = 0, a_lo = 0;
    double alpha = -1;
    ~PrPlan() {
        blocks.release(); outdeg.release(); contrib.release(); partials.release();
        ctl.release(); dang.release(); segbase.release(); seg_range.release(); segs.release();
    }
};

// Row blocks over the CSC offsets: consecutive rows while the block holds at
// most kNnz in-edges and kRows rows; a longer row forms a block of its own.
static int build_pr_plan(olv_graph *g, PrPlan &p) {
    const uint32_t V = g->V;
    std::vector<uint32_t> cp(V + 1);
    OLV_CUDA(cudaMemcpyAsync(cp.data(), g->colptr.p, ((size_t)V + 1) * 4, cudaMemcpyDeviceToHost,
                             g->stream));
    OLV_CUDA(cudaStreamSynchronize(g->stream));
    std::vector<uint32_t> b;
    b.reserve(g->E / kNnz + V / kRows + 16);
    uint32_t v = 0;
    b.push_back(0);
    while (v < V) {
        const uint32_t start = v;
        if (cp[v + 1] - cp[v] > kNnz) {
            v++;
        } else {
            while (v < V && v - start < kRows && cp[v + 1] - cp[start] <= kNnz) v++;
        }
        b.push_back(v);
    }
    p.nblocks = (uint32_t)b.size() - 1;
    // long rows (one per block) are cut into kSeg-edge segments
    std::vector<uint32_t> segbase(p.nblocks, 0xffffffffu);
    std::vector<uint2> ranges;
    for (uint32_t k = 0; k < p.nblocks; k++) {
        const uint32_t e0 = cp[b[k]], e1 = cp[b[k + 1]];
        if (e1 - e0 <= kNnz) continue;
        segbase[k] = (uint32_t)ranges.size();
        for (uint32_t x = e0; x < e1; x += kSeg) ranges.push_back(make_uint2(x, std::min(e1, x + kSeg)));
    }
    p.nsegs = (uint32_t)ranges.size();
    OLV_TRY(p.segbase.ensure(segbase.size() * 4 + 16));
    OLV_TRY(p.seg_range.ensure(ranges.size() * 8 + 16));
    OLV_TRY(p.segs.ensure(ranges.size() * 8 + 16));
    OLV_CUDA(cudaMemcpyAsync(p.segbase.p, segbase.data(), segbase.size() * 4,
                             cudaMemcpyHostToDevice, g->stream));
    if (!ranges.empty())
        OLV_CUDA(cudaMemcpyAsync(p.seg_range.p, ranges.data(), ranges.size() * 8,
                                 cudaMemcpyHostToDevice, g->stream));
    OLV_TRY(p.blocks.ensure(b.size() * 4));
    OLV_CUDA(cudaMemcpyAsync(p.blocks.p, b.data(), b.size() * 4, cudaMemcpyHostToDevice,
                             g->stream));
    OLV_TRY(p.outdeg.ensure((size_t)V * 4 + 16));
    k_outdeg<<<g->num_sms * 8, kBlock, 0, g->stream>>>(g->rowptr.as<uint32_t>(), V,
                                                      p.outdeg.as<uint32_t>());
    OLV_TRY(p.contrib.ensure((size_t)V * 8 + 32));
    OLV_TRY(p.partials.ensure((size_t)p.nblocks * 16 + 16));
    OLV_TRY(p.ctl.ensure(sizeof(PrCtl)));
    OLV_TRY(p.dang.ensure(16));
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaStreamSynchronize(g->stream));
    return OLV_OK;
}

template <class Sink>
static int pr_iteration(olv_graph *g, PrPlan &p, float *rank, Sink &&sink,
                        cudaGraphConditionalHandle h, int use_cond) {
    const uint32_t *colptr = g->colptr.as<uint32_t>();
    const uint32_t *rowidx = g->rowidx.as<uint32_t>();
    const uint32_t *blocks = p.blocks.as<uint32_t>();
    const uint32_t *outdeg = p.outdeg.as<uint32_t>();
    const float *c0 = p.contrib.as<float>();
    const float *c1 = p.contrib.as<float>() + g->V;
    PrCtl *ctl = p.ctl.as<PrCtl>();
    double *partials = p.partials.as<double>();
    float a_hi = p.a_hi, a_lo = p.a_lo;
    uint32_t nparts = p.nblocks;
    const uint32_t *segbase = p.segbase.as<uint32_t>();
    const uint2 *seg_range = p.seg_range.as<uint2>();
    float2 *segs = p.segs.as<float2>();
    const float2 *csegs = segs;
    const PrCtl *cctl = ctl;
    if (p.nsegs) {
        void *a_seg[] = {&rowidx, &seg_range, &c0, &c1, &cctl, &segs};
        OLV_TRY(sink((const void *)k_pr_segments, dim3(p.nsegs), dim3(kBlock), a_seg));
    }
    void *a_pull[] = {&colptr, &rowidx, &blocks, &outdeg, &c0, &c1, &rank, &ctl, &partials,
                      &a_hi, &a_lo, &segbase, &csegs};
    OLV_TRY(sink((const void *)k_pr_pull, dim3(p.nblocks), dim3(kBlock), a_pull));
    const double *cpart = partials;
    void *a_red[] = {&ctl, &cpart, &nparts, &h, &use_cond};
    OLV_TRY(sink((const void *)k_pr_reduce, dim3(1), dim3(kRedThreads), a_red));
    return OLV_OK;
}

}  // namespace olv

using namespace olv;

struct PrState {
    PrPlan plan;
    WhileGraph graph;
    float *graph_rank = nullptr;
};

static PrState *pr_state(olv_graph *g) { return static_cast<PrState *>(g->pr_state); }

void olv::release_pr_state(olv_graph *g) {
    PrState *s = pr_state(g);
    if (s) {
        s->graph.destroy();
        delete s;
    }
    g->pr_state = nullptr;
}

extern "C" int olv_pagerank(olv_graph *g, double alpha, int max_it, double tol, int dangling_mode,
                            float *rank_out, olv_stats *st) {
    OLV_CHECK_ARG(g && rank_out, "olv_pagerank: null pointer");
    OLV_CHECK_ARG(alpha >= 0.0 && alpha < 1.0, "olv_pagerank: alpha must be in [0,1)");
    OLV_CHECK_ARG(max_it >= 0, "olv_pagerank: max_it must be >= 0");
    OLV_CHECK_ARG(dangling_mode == OLV_DANGLING_UNIFORM || dangling_mode == OLV_DANGLING_LEAK,
                  "olv_pagerank: bad dangling_mode %d", dangling_mode);
    cudaStream_t s = g->stream;
    PrState *ps = pr_state(g);
    if (!ps) {
        ps = new PrState();
        g->pr_state = ps;
        int r = build_pr_plan(g, ps->plan);
        if (r != OLV_OK) {
            release_pr_state(g);
            return r;
        }
    }
    PrPlan &p = ps->plan;
    // alpha as an unevaluated FP32 pair so the update carries FP64-level alpha
    const double ad = alpha;
    p.a_hi = (float)ad;
    p.a_lo = (float)(ad - (double)p.a_hi);
    const bool dev_out = is_device_ptr(rank_out);
    if (!dev_out) OLV_TRY(g->ws.level.ensure((size_t)g->V * 4 + 16));
    float *rank = dev_out ? rank_out : g->ws.level.as<float>();

    OLV_CUDA(cudaEventRecord(g->ev0, s));
    OLV_CUDA(cudaMemsetAsync(p.dang.p, 0, 8, s));
    k_pr_init<<<g->num_sms * 8, kBlock, 0, s>>>(p.outdeg.as<uint32_t>(), g->V, rank,
                                               p.contrib.as<float>(),
                                               p.dang.as<unsigned long long>());
    k_pr_ctl_init<<<1, 1, 0, s>>>(p.ctl.as<PrCtl>(), p.dang.as<unsigned long long>(), g->V, ad,
                                  (uint32_t)max_it, tol,
                                  dangling_mode == OLV_DANGLING_LEAK ? 1u : 0u);
    OLV_CUDA(cudaGetLastError());
    bool launched = false;
    if (g->tune.use_graphs && max_it > 0) {
        if (!ps->graph.ready || ps->graph_rank != rank) {
            int r = ps->graph.begin();
            auto sink = [&](const void *f, dim3 gr, dim3 bl, void **args) {
                return ps->graph.add(f, gr, bl, args);
            };
            if (r == OLV_OK) r = pr_iteration(g, p, rank, sink, ps->graph.handle, 1);
            if (r == OLV_OK) r = ps->graph.finish();
            ps->graph_rank = rank;
            if (r != OLV_OK) ps->graph.destroy();
        }
        if (ps->graph.ready) {
            OLV_TRY(ps->graph.launch(s));
            launched = true;
        }
    }
    if (!launched) {
        auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
            OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
            return OLV_OK;
        };
        for (int it = 0; it < max_it; it++) OLV_TRY(pr_iteration(g, p, rank, launch, 0, 0));
    }
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    PrCtl hc;
    OLV_CUDA(cudaMemcpyAsync(&hc, p.ctl.p, sizeof(PrCtl), cudaMemcpyDeviceToHost, s));
    if (!dev_out)
        OLV_CUDA(cudaMemcpyAsync(rank_out, rank, (size_t)g->V * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    if (st) {
        float ms = 0;
        OLV_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        st->iterations = hc.iter;
        st->pull_steps = 0;
        st->vertices_reached = g->V;
        st->edges_traversed = g->E * (uint64_t)hc.iter;
        st->edges_relaxed = g->E * (uint64_t)hc.iter;
        st->residual = hc.residual;
        st->device_ms = ms;
    }
    return OLV_OK;
}
