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
//   * the solve runs on a relabelled copy of the reverse graph (CSC): vertices
//     renumbered by in-degree, longest rows first (olv_rowtiles.cuh), built
//     once per graph.  Ranks, contributions r/outdeg and out-degrees live in
//     the new order; the ranks are mapped back to the caller's ids once, at
//     the end of the solve;
//   * each iteration is one pull pass over the in-edges: a group of 1..32
//     lanes per row (by row length) sums the row's contributions in a fixed
//     order with compensated (two-sum) FP32 arithmetic, so results do not
//     depend on scheduling and carry ~1 rounding per vertex; rows longer than
//     kTileLong are summed in fixed segments first;
//   * the same pass writes the next iteration's contributions r/outdeg and
//     per-CTA FP64 partial sums of |r' - r| and of the dangling mass;
//   * a one-CTA kernel folds the partials in a fixed order (FP64), decides
//     convergence on the device and sets the loop condition of the CUDA graph
//     that runs all iterations.
#include <algorithm>
#include <vector>

#include "olive_b200/olv_advance.cuh"
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"
#include "olv_rowtiles.cuh"

namespace olv {

constexpr int kRedThreads = 1024;

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

// r' = alpha * (s + c) + base, with alpha split into hi + lo FP32 parts.
__device__ __forceinline__ float pr_update(float s, float c, float a_hi, float a_lo, float base) {
    const float t = fmaf(a_lo, s, fmaf(a_hi, c, base));
    return fmaf(a_hi, s, t);
}

// Row sums over in-edges of the contributions r[u]/outdeg(u); the row update
// writes the rank, the next contribution and FP64 |r'-r| / dangling partials.
struct PrOp {
    const uint32_t *done;
    const PrCtl *ctl;
    const float *c0, *c1;
    float *rank;
    const uint32_t *outdeg;
    float a_hi, a_lo;
    const float *cin;
    float *cout;
    float base;

    __device__ __forceinline__ void begin() {
        const bool odd = ctl->iter & 1;
        cin = odd ? c1 : c0;
        cout = const_cast<float *>(odd ? c0 : c1);
        base = (float)ctl->base;
    }
    __device__ __forceinline__ float term(uint32_t, uint32_t j) const { return __ldg(&cin[j]); }
    struct Row {
        float old;       // rank before this iteration
        uint32_t deg;    // out-degree
    };
    __device__ __forceinline__ Row row(uint32_t v) const { return Row{rank[v], __ldg(&outdeg[v])}; }
    __device__ __forceinline__ void finish(uint32_t v, float s, float c, const Row &r, double &res,
                                           double &dang) const {
        const float nr = pr_update(s, c, a_hi, a_lo, base);
        rank[v] = nr;
        res += fabs((double)nr - (double)r.old);
        if (r.deg) {
            cout[v] = __fdiv_rn(nr, (float)r.deg);
        } else {
            cout[v] = 0.0f;
            dang += (double)nr;
        }
    }
};

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

// out-degree of every vertex, in the relabelled order
__global__ void k_outdeg_perm(const uint32_t *__restrict__ rowptr,
                              const uint32_t *__restrict__ perm, uint32_t V, uint32_t *d) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = perm[i];
        d[i] = rowptr[v + 1] - rowptr[v];
    }
}

// rank[v] = rank of v's new id (coalesced writes, gathers from an L2-sized array)
__global__ void k_pr_unpermute(const float *__restrict__ rank_new,
                               const uint32_t *__restrict__ newid, uint32_t V,
                               float *__restrict__ rank) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x)
        rank[v] = rank_new[newid[v]];
}

// ------------------------------------------------------------------ host --
struct PrPlan {
    TilePlan tp;
    DevBuf outdeg, contrib, rank, ctl, dang;   // outdeg, contrib, rank: new order
    float a_hi = 0, a_lo = 0;
    ~PrPlan() {
        tp.release(); outdeg.release(); contrib.release(); rank.release(); ctl.release();
        dang.release();
    }
};

static int build_pr_plan(olv_graph *g, PrPlan &p) {
    const uint32_t V = g->V;
    OLV_TRY(build_tile_plan(g->colptr.as<uint32_t>(), g->rowidx.as<uint32_t>(), V, g->stream,
                            p.tp, true, g->tune.pr_tile_u));
    OLV_TRY(p.outdeg.ensure((size_t)V * 4 + 16));
    k_outdeg_perm<<<g->num_sms * 8, kBlock, 0, g->stream>>>(
        g->rowptr.as<uint32_t>(), p.tp.perm.as<uint32_t>(), V, p.outdeg.as<uint32_t>());
    OLV_TRY(p.contrib.ensure((size_t)V * 8 + 32));
    OLV_TRY(p.rank.ensure((size_t)V * 4 + 16));
    OLV_TRY(p.ctl.ensure(sizeof(PrCtl)));
    OLV_TRY(p.dang.ensure(16));
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaStreamSynchronize(g->stream));
    return OLV_OK;
}

template <class Sink>
static int pr_iteration(olv_graph *g, PrPlan &p, Sink &&sink, cudaGraphConditionalHandle h,
                        int use_cond) {
    PrCtl *ctl = p.ctl.as<PrCtl>();
    PrOp op;
    op.done = &ctl->done;
    op.ctl = ctl;
    op.c0 = p.contrib.as<float>();
    op.c1 = p.contrib.as<float>() + g->V;
    op.rank = p.rank.as<float>();
    op.outdeg = p.outdeg.as<uint32_t>();
    op.a_hi = p.a_hi;
    op.a_lo = p.a_lo;
    op.cin = nullptr;
    op.cout = nullptr;
    op.base = 0;
    OLV_TRY(tile_pass(p.tp, op, sink));
    const double *cpart = p.tp.partials.as<double>();
    uint32_t nparts = kTileCTAs;
    void *a_red[] = {&ctl, &cpart, &nparts, &h, &use_cond};
    OLV_TRY(sink((const void *)k_pr_reduce, dim3(1), dim3(kRedThreads), a_red));
    return OLV_OK;
}

}  // namespace olv

using namespace olv;

struct PrState {
    PrPlan plan;
    WhileGraph graph;
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
    float *rank_new = p.rank.as<float>();

    OLV_CUDA(cudaEventRecord(g->ev0, s));
    OLV_CUDA(cudaMemsetAsync(p.dang.p, 0, 8, s));
    k_pr_init<<<g->num_sms * 8, kBlock, 0, s>>>(p.outdeg.as<uint32_t>(), g->V, rank_new,
                                               p.contrib.as<float>(),
                                               p.dang.as<unsigned long long>());
    k_pr_ctl_init<<<1, 1, 0, s>>>(p.ctl.as<PrCtl>(), p.dang.as<unsigned long long>(), g->V, ad,
                                  (uint32_t)max_it, tol,
                                  dangling_mode == OLV_DANGLING_LEAK ? 1u : 0u);
    OLV_CUDA(cudaGetLastError());
    bool launched = false;
    if (g->tune.use_graphs && max_it > 0) {
        if (!ps->graph.ready) {
            int r = ps->graph.begin();
            auto sink = [&](const void *f, dim3 gr, dim3 bl, void **args) {
                return ps->graph.add(f, gr, bl, args);
            };
            if (r == OLV_OK) r = pr_iteration(g, p, sink, ps->graph.handle, 1);
            if (r == OLV_OK) r = ps->graph.finish();
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
        for (int it = 0; it < max_it; it++) OLV_TRY(pr_iteration(g, p, launch, 0, 0));
    }
    k_pr_unpermute<<<g->num_sms * 8, kBlock, 0, s>>>(rank_new, p.tp.newid.as<uint32_t>(), g->V,
                                                    rank);
    OLV_CUDA(cudaGetLastError());
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
