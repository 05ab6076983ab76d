// Differentiable weighted PageRank (no reference counterpart).
//
//   W_u = sum_v w_uv,  P_uv = w_uv / W_u  (rows without out-edges are zero)
//   forward:  r = (1-alpha) p + alpha P^T r        (pull over the CSC)
//   adjoint:  lambda = g + alpha P lambda           (pull over the CSR: the
//             same row-sum engine over the reversed edges)
//   dL/dw_uv = alpha r_u (lambda_v - t_u) / W_u,   t_u = sum_x P_ux lambda_x
//   dL/dp    = (1-alpha) lambda                     for L = sum_v g_v r_v.
// Both solves are Jacobi sweeps with deterministic compensated FP32 row sums
// and FP64 residual norms, run as CUDA graphs; the gradient is implicit at the
// fixed point, so memory is O(V + E) with no tape.
//
// The row sums run on row-reordered copies of the CSC (forward) and the CSR
// (adjoint, W, t): rows sorted by length so that a group of 1..32 lanes per
// row fits every row of a warp (olv_rowtiles.cuh); neighbour ids and all
// per-vertex arrays keep the caller's numbering, and the edge weights are
// permuted into each copy's entry order at the start of every forward solve.
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"
#include "olv_rowtiles.cuh"

struct olv_wpr_ctx {
    olv_graph *g = nullptr;
    double alpha = 0.85;
    float a_hi = 0, a_lo = 0;
    olv::DevBuf W, r, s2, tp, lam2, t, gbuf;   // r: [V]; s2: 2V; lam2: 2V
    olv::DevBuf ctl;                           // IterCtl
    olv::WhileGraph fwd, bwd;
    double fwd_alpha = -1, bwd_alpha = -1;
};

namespace olv {

struct WprPlans {
    RowPlan csr;               // row blocks of the CSR (gradient kernels)
    TilePlan tcsc, tcsr;       // row-reordered CSC and CSR (row sums)
    DevBuf wc, wr;             // weights in tcsc / tcsr entry order
    ~WprPlans() {
        csr.release();
        tcsc.release();
        tcsr.release();
        wc.release();
        wr.release();
    }
};

// --- row-sum ops ---------------------------------------------------------
struct WsumOp {   // W_u = sum of out-weights (CSR)
    const uint32_t *done;
    const float *w;
    float *W;
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ float term(uint32_t e, uint32_t) const { return __ldg(&w[e]); }
    struct Row {
        uint32_t unused;
    };
    __device__ __forceinline__ Row row(uint32_t) const { return Row{0}; }
    __device__ __forceinline__ void finish(uint32_t u, float s, float c, const Row &, double &,
                                           double &) const {
        W[u] = s + c;
    }
};

struct WfwdOp {   // r'[v] = (1-alpha) p[v] + alpha sum_{u->v} w_uv r[u]/W_u
    const uint32_t *done;
    const IterCtl *ctl;
    const float *wc;      // CSC-ordered weights
    const float *s0, *s1; // r/W ping-pong
    const float *W, *tp;  // tp = (1-alpha) p
    float *r;
    float a_hi, a_lo;
    const float *sin;
    float *sout;
    __device__ __forceinline__ void begin() {
        const bool odd = ctl->iter & 1;
        sin = odd ? s1 : s0;
        sout = const_cast<float *>(odd ? s0 : s1);
    }
    __device__ __forceinline__ float term(uint32_t e, uint32_t u) const {
        return __ldg(&wc[e]) * __ldg(&sin[u]);
    }
    struct Row {
        float tp, r, W;
    };
    __device__ __forceinline__ Row row(uint32_t v) const { return Row{tp[v], r[v], W[v]}; }
    __device__ __forceinline__ void finish(uint32_t v, float s, float c, const Row &q, double &res,
                                           double &) const {
        const float t = fmaf(a_lo, s, fmaf(a_hi, c, q.tp));
        const float nr = fmaf(a_hi, s, t);
        res += fabs((double)nr - (double)q.r);
        r[v] = nr;
        sout[v] = q.W > 0.0f ? __fdiv_rn(nr, q.W) : 0.0f;
    }
};

struct WadjOp {   // lambda'[u] = g[u] + alpha sum_{u->v} w_uv lambda[v] / W_u
    const uint32_t *done;
    const IterCtl *ctl;
    const float *w;        // CSR weights
    const float *l0, *l1;  // lambda ping-pong
    const float *W, *gv;
    float *t;              // t_u of the sweep (for the gradient)
    float a_hi, a_lo;
    const float *lin;
    float *lout;
    __device__ __forceinline__ void begin() {
        const bool odd = ctl->iter & 1;
        lin = odd ? l1 : l0;
        lout = const_cast<float *>(odd ? l0 : l1);
    }
    __device__ __forceinline__ float term(uint32_t e, uint32_t v) const {
        return __ldg(&w[e]) * __ldg(&lin[v]);
    }
    struct Row {
        float W, g, lam;
    };
    __device__ __forceinline__ Row row(uint32_t u) const { return Row{W[u], gv[u], lin[u]}; }
    __device__ __forceinline__ void finish(uint32_t u, float s, float c, const Row &q, double &res,
                                           double &) const {
        const float tu = q.W > 0.0f ? __fdiv_rn(s + c, q.W) : 0.0f;
        const float nl = fmaf(a_hi, tu, fmaf(a_lo, tu, q.g));
        res += fabs((double)nl - (double)q.lam);
        lout[u] = nl;
        t[u] = tu;
    }
};

struct WtOp {     // t_u from the final lambda, and dL/dp = (1-alpha) lambda
    const uint32_t *done;
    const float *w, *lam, *W;
    float *t, *dp;
    float one_minus_alpha;
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ float term(uint32_t e, uint32_t v) const {
        return __ldg(&w[e]) * __ldg(&lam[v]);
    }
    struct Row {
        float W, lam;
    };
    __device__ __forceinline__ Row row(uint32_t u) const { return Row{W[u], lam[u]}; }
    __device__ __forceinline__ void finish(uint32_t u, float s, float c, const Row &q, double &,
                                           double &) const {
        t[u] = q.W > 0.0f ? __fdiv_rn(s + c, q.W) : 0.0f;
        if (dp) dp[u] = one_minus_alpha * q.lam;
    }
};

// dL/dw_e for the CSR edges of a row block (rows found by binary search in
// shared memory), or of one long-row segment.
__global__ void __launch_bounds__(kBlock)
k_wpr_grad_blocks(const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ col,
                  const uint32_t *__restrict__ blocks, const float *__restrict__ r,
                  const float *__restrict__ W, const float *__restrict__ lam,
                  const float *__restrict__ t, float alpha, float *__restrict__ dw) {
    const uint32_t r0 = blocks[blockIdx.x], r1 = blocks[blockIdx.x + 1];
    const uint32_t e0 = ptr[r0], e1 = ptr[r1];
    if (e1 - e0 > kNnz) return;   // long rows: k_wpr_grad_segments
    __shared__ uint32_t s_ptr[kRows + 1];
    const uint32_t nr = r1 - r0;
    for (uint32_t i = threadIdx.x; i <= nr; i += kBlock) s_ptr[i] = ptr[r0 + i];
    __syncthreads();
    for (uint32_t e = e0 + threadIdx.x; e < e1; e += kBlock) {
        uint32_t lo = 0, hi = nr;   // largest k with s_ptr[k] <= e
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_ptr[mid] <= e) lo = mid; else hi = mid;
        }
        const uint32_t u = r0 + lo;
        const float Wu = W[u];
        const float coef = Wu > 0.0f ? __fdiv_rn(alpha * r[u], Wu) : 0.0f;
        dw[e] = coef * (__ldg(&lam[col[e]]) - t[u]);
    }
}

__global__ void __launch_bounds__(kBlock)
k_wpr_grad_segments(const uint32_t *__restrict__ col, const uint2 *__restrict__ seg_range,
                    const uint32_t *__restrict__ seg_row, const float *__restrict__ r,
                    const float *__restrict__ W, const float *__restrict__ lam,
                    const float *__restrict__ t, float alpha, float *__restrict__ dw) {
    const uint2 sr = seg_range[blockIdx.x];
    const uint32_t u = seg_row[blockIdx.x];
    const float Wu = W[u];
    const float coef = Wu > 0.0f ? __fdiv_rn(alpha * r[u], Wu) : 0.0f;
    const float tu = t[u];
    for (uint32_t e = sr.x + threadIdx.x; e < sr.y; e += kBlock)
        dw[e] = coef * (__ldg(&lam[col[e]]) - tu);
}

__global__ void k_wpr_init(uint32_t V, const float *p, const float *W, float alpha, float *tp,
                           float *r, float *s0) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        const float pv = p[v];
        tp[v] = (1.0f - alpha) * pv;
        r[v] = pv;
        s0[v] = W[v] > 0.0f ? __fdiv_rn(pv, W[v]) : 0.0f;
    }
}

__global__ void k_copy_f32(const float *__restrict__ a, float *__restrict__ b, uint32_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

__global__ void k_iter_init(IterCtl *c, uint32_t max_it, double tol) {
    IterCtl t = {};
    t.max_it = max_it;
    t.tol = tol;
    t.done = max_it == 0;
    *c = t;
}

static WprPlans *wpr_plans(olv_graph *g) { return static_cast<WprPlans *>(g->wpr_state); }

static int ensure_wpr_plans(olv_graph *g) {
    if (g->wpr_state) return OLV_OK;
    WprPlans *p = new WprPlans();
    int r = build_row_plan(g->rowptr.as<uint32_t>(), g->V, g->stream, p->csr);
    if (r == OLV_OK)
        r = build_tile_plan(g->colptr.as<uint32_t>(), g->rowidx.as<uint32_t>(), g->V, g->stream,
                            p->tcsc, false, g->tune.pr_tile_u);
    if (r == OLV_OK)
        r = build_tile_plan(g->rowptr.as<uint32_t>(), g->col.as<uint32_t>(), g->V, g->stream,
                            p->tcsr, false, g->tune.pr_tile_u);
    if (r == OLV_OK) r = p->wc.ensure(g->E * 4 + 16);
    if (r == OLV_OK) r = p->wr.ensure(g->E * 4 + 16);
    if (r != OLV_OK) {
        delete p;
        return r;
    }
    g->wpr_state = p;
    return OLV_OK;
}

void release_wpr_state(olv_graph *g) {
    delete wpr_plans(g);
    g->wpr_state = nullptr;
}

static void split_alpha(double alpha, float &hi, float &lo) {
    hi = (float)alpha;
    lo = (float)(alpha - (double)hi);
}

static int copy_vec_in(DevBuf &dst, const float *src, size_t n, cudaStream_t s) {
    OLV_TRY(dst.ensure(n * 4 + 16));
    OLV_CUDA(cudaMemcpyAsync(dst.p, src, n * 4, cudaMemcpyDefault, s));
    return OLV_OK;
}

}  // namespace olv

using namespace olv;

extern "C" int olv_wpr_forward(olv_graph *g, const float *w, const float *p, double alpha,
                               int max_it, double tol, float *r_out, olv_wpr_ctx **ctx_out,
                               olv_stats *st) {
    OLV_CHECK_ARG(g && p && ctx_out, "olv_wpr_forward: null pointer");
    OLV_CHECK_ARG(alpha >= 0 && alpha < 1 && max_it >= 0, "olv_wpr_forward: bad alpha / max_it");
    if (w) OLV_TRY(olv_graph_set_weights_f32(g, w));
    OLV_CHECK_ARG(g->weight_type == OLV_W_F32, "olv_wpr_forward: graph has no FP32 weights");
    OLV_TRY(ensure_wpr_plans(g));
    WprPlans &pl = *wpr_plans(g);
    olv_wpr_ctx *c = *ctx_out;
    if (!c) {
        c = new (std::nothrow) olv_wpr_ctx();
        if (!c) {
            set_error("olv_wpr_forward: host allocation failed");
            return OLV_ERR_NOMEM;
        }
        *ctx_out = c;
    }
    OLV_CHECK_ARG(c->g == nullptr || c->g == g, "olv_wpr_forward: context belongs to another graph");
    c->g = g;
    c->alpha = alpha;
    split_alpha(alpha, c->a_hi, c->a_lo);
    const size_t V = g->V;
    cudaStream_t s = g->stream;
    OLV_TRY(c->W.ensure(V * 4 + 16));
    OLV_TRY(c->r.ensure(V * 4 + 16));
    OLV_TRY(c->s2.ensure(V * 8 + 32));
    OLV_TRY(c->tp.ensure(V * 4 + 16));
    OLV_TRY(c->ctl.ensure(sizeof(IterCtl)));
    OLV_TRY(copy_vec_in(c->gbuf, p, V, s));   // p staged in gbuf during the forward
    IterCtl *ctl = c->ctl.as<IterCtl>();
    OLV_CUDA(cudaEventRecord(g->ev0, s));
    // the weights in the entry orders of the two row-reordered copies
    k_permute_entries<<<g->num_sms * 8, kBlock, 0, s>>>(g->csc_w.as<float>(),
                                                       pl.tcsc.pos.as<uint32_t>(), g->E,
                                                       pl.wc.as<float>());
    k_permute_entries<<<g->num_sms * 8, kBlock, 0, s>>>(g->w.as<float>(),
                                                       pl.tcsr.pos.as<uint32_t>(), g->E,
                                                       pl.wr.as<float>());
    // W = row sums of the weights (one pass, same deterministic engine)
    {
        k_iter_init<<<1, 1, 0, s>>>(ctl, 1, 0.0);   // done = 0 for the single pass
        PermOp<WsumOp> op{WsumOp{&ctl->done, pl.wr.as<float>(), c->W.as<float>()},
                          pl.tcsr.perm.as<uint32_t>(), &ctl->done};
        auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
            OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
            return OLV_OK;
        };
        OLV_TRY(tile_pass(pl.tcsr, op, launch));
    }
    k_wpr_init<<<g->num_sms * 8, kBlock, 0, s>>>(g->V, c->gbuf.as<float>(), c->W.as<float>(),
                                                (float)alpha, c->tp.as<float>(), c->r.as<float>(),
                                                c->s2.as<float>());
    k_iter_init<<<1, 1, 0, s>>>(ctl, (uint32_t)max_it, tol);
    OLV_CUDA(cudaGetLastError());
    WfwdOp fop;
    WfwdOp &op = fop;
    op.done = &ctl->done;
    op.ctl = ctl;
    op.wc = pl.wc.as<float>();
    op.s0 = c->s2.as<float>();
    op.s1 = c->s2.as<float>() + V;
    op.W = c->W.as<float>();
    op.tp = c->tp.as<float>();
    op.r = c->r.as<float>();
    op.a_hi = c->a_hi;
    op.a_lo = c->a_lo;
    op.sin = nullptr;
    op.sout = nullptr;
    PermOp<WfwdOp> pop{fop, pl.tcsc.perm.as<uint32_t>(), &ctl->done};
    const double *cpart = pl.tcsc.partials.as<double>();
    uint32_t nparts = kTileCTAs;
    auto body = [&](auto &&sink, cudaGraphConditionalHandle h, int use_cond) {
        OLV_TRY(tile_pass(pl.tcsc, pop, sink));
        void *a_fold[] = {&ctl, &cpart, &nparts, &h, &use_cond};
        return sink((const void *)k_iter_fold, dim3(1), dim3(kFoldThreads), a_fold);
    };
    bool launched = false;
    if (c->fwd.ready && c->fwd_alpha != alpha) c->fwd.destroy();
    if (g->tune.use_graphs && max_it > 0) {
        if (!c->fwd.ready) {
            c->fwd_alpha = alpha;
            int r = c->fwd.begin();
            auto sink = [&](const void *f, dim3 gr, dim3 bl, void **args) {
                return c->fwd.add(f, gr, bl, args);
            };
            if (r == OLV_OK) r = body(sink, c->fwd.handle, 1);
            if (r == OLV_OK) r = c->fwd.finish();
            if (r != OLV_OK) c->fwd.destroy();
        }
        if (c->fwd.ready) {
            OLV_TRY(c->fwd.launch(s));
            launched = true;
        }
    }
    if (!launched) {
        auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
            OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
            return OLV_OK;
        };
        for (int i = 0; i < max_it; i++) OLV_TRY(body(launch, 0, 0));
    }
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    IterCtl hc;
    OLV_CUDA(cudaMemcpyAsync(&hc, ctl, sizeof hc, cudaMemcpyDeviceToHost, s));
    if (r_out) OLV_CUDA(cudaMemcpyAsync(r_out, c->r.p, V * 4, cudaMemcpyDefault, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    if (st) {
        float ms = 0;
        OLV_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        st->iterations = hc.iter;
        st->pull_steps = 0;
        st->vertices_reached = V;
        st->edges_traversed = g->E * (uint64_t)hc.iter;
        st->edges_relaxed = st->edges_traversed;
        st->residual = hc.residual;
        st->device_ms = ms;
    }
    return OLV_OK;
}

extern "C" int olv_wpr_backward(olv_wpr_ctx *c, const float *gvec, int max_it, double tol,
                                float *dw_out, float *dp_out, olv_stats *st) {
    OLV_CHECK_ARG(c && c->g && gvec && dw_out, "olv_wpr_backward: null pointer or no forward");
    OLV_CHECK_ARG(max_it >= 0, "olv_wpr_backward: bad max_it");
    olv_graph *g = c->g;
    if (!wpr_plans(g)) {   // the row plans were dropped (pr_tile_u changed) since the forward
        set_error("olv_wpr_backward: the graph's row plans changed since olv_wpr_forward; "
                  "run the forward again");
        return OLV_ERR_STATE;
    }
    WprPlans &pl = *wpr_plans(g);
    const size_t V = g->V;
    const uint64_t E = g->E;
    cudaStream_t s = g->stream;
    OLV_TRY(c->lam2.ensure(V * 8 + 32));
    OLV_TRY(c->t.ensure(V * 4 + 16));
    OLV_TRY(copy_vec_in(c->gbuf, gvec, V, s));
    const bool dev_dw = is_device_ptr(dw_out);
    const bool dev_dp = dp_out && is_device_ptr(dp_out);
    DevBuf dwbuf, dpbuf;
    if (!dev_dw) OLV_TRY(dwbuf.ensure(E * 4 + 16));
    if (dp_out && !dev_dp) OLV_TRY(dpbuf.ensure(V * 4 + 16));
    float *dw = dev_dw ? dw_out : dwbuf.as<float>();
    float *dp = dp_out ? (dev_dp ? dp_out : dpbuf.as<float>()) : nullptr;
    IterCtl *ctl = c->ctl.as<IterCtl>();
    OLV_CUDA(cudaEventRecord(g->ev0, s));
    k_copy_f32<<<g->num_sms * 8, kBlock, 0, s>>>(c->gbuf.as<float>(), c->lam2.as<float>(), g->V);
    k_iter_init<<<1, 1, 0, s>>>(ctl, (uint32_t)max_it, tol);
    OLV_CUDA(cudaGetLastError());
    WadjOp aop;
    WadjOp &op = aop;
    op.done = &ctl->done;
    op.ctl = ctl;
    op.w = pl.wr.as<float>();
    op.l0 = c->lam2.as<float>();
    op.l1 = c->lam2.as<float>() + V;
    op.W = c->W.as<float>();
    op.gv = c->gbuf.as<float>();
    op.t = c->t.as<float>();
    op.a_hi = c->a_hi;
    op.a_lo = c->a_lo;
    op.lin = nullptr;
    op.lout = nullptr;
    PermOp<WadjOp> pop{aop, pl.tcsr.perm.as<uint32_t>(), &ctl->done};
    const double *cpart = pl.tcsr.partials.as<double>();
    uint32_t nparts = kTileCTAs;
    auto body = [&](auto &&sink, cudaGraphConditionalHandle h, int use_cond) {
        OLV_TRY(tile_pass(pl.tcsr, pop, sink));
        void *a_fold[] = {&ctl, &cpart, &nparts, &h, &use_cond};
        return sink((const void *)k_iter_fold, dim3(1), dim3(kFoldThreads), a_fold);
    };
    bool launched = false;
    if (c->bwd.ready && c->bwd_alpha != c->alpha) c->bwd.destroy();
    if (g->tune.use_graphs && max_it > 0) {
        if (!c->bwd.ready) {
            c->bwd_alpha = c->alpha;
            int r = c->bwd.begin();
            auto sink = [&](const void *f, dim3 gr, dim3 bl, void **args) {
                return c->bwd.add(f, gr, bl, args);
            };
            if (r == OLV_OK) r = body(sink, c->bwd.handle, 1);
            if (r == OLV_OK) r = c->bwd.finish();
            if (r != OLV_OK) c->bwd.destroy();
        }
        if (c->bwd.ready) {
            OLV_TRY(c->bwd.launch(s));
            launched = true;
        }
    }
    if (!launched) {
        auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
            OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
            return OLV_OK;
        };
        for (int i = 0; i < max_it; i++) OLV_TRY(body(launch, 0, 0));
    }
    IterCtl hc;
    OLV_CUDA(cudaMemcpyAsync(&hc, ctl, sizeof hc, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    // final lambda lives in the buffer the last sweep wrote
    const float *lam = c->lam2.as<float>() + ((hc.iter & 1) ? V : 0);
    {
        k_iter_init<<<1, 1, 0, s>>>(ctl, 1, 0.0);
        PermOp<WtOp> top{WtOp{&ctl->done, pl.wr.as<float>(), lam, c->W.as<float>(),
                              c->t.as<float>(), dp, (float)(1.0 - c->alpha)},
                         pl.tcsr.perm.as<uint32_t>(), &ctl->done};
        auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
            OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
            return OLV_OK;
        };
        OLV_TRY(tile_pass(pl.tcsr, top, launch));
    }
    k_wpr_grad_blocks<<<pl.csr.nblocks, kBlock, 0, s>>>(
        g->rowptr.as<uint32_t>(), g->col.as<uint32_t>(), pl.csr.blocks.as<uint32_t>(),
        c->r.as<float>(), c->W.as<float>(), lam, c->t.as<float>(), (float)c->alpha, dw);
    if (pl.csr.nsegs)
        k_wpr_grad_segments<<<pl.csr.nsegs, kBlock, 0, s>>>(
            g->col.as<uint32_t>(), pl.csr.seg_range.as<uint2>(), pl.csr.seg_row.as<uint32_t>(),
            c->r.as<float>(), c->W.as<float>(), lam, c->t.as<float>(), (float)c->alpha, dw);
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    if (!dev_dw) OLV_CUDA(cudaMemcpyAsync(dw_out, dw, E * 4, cudaMemcpyDeviceToHost, s));
    if (dp_out && !dev_dp) OLV_CUDA(cudaMemcpyAsync(dp_out, dp, V * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    if (st) {
        float ms = 0;
        OLV_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        st->iterations = hc.iter;
        st->pull_steps = 0;
        st->vertices_reached = V;
        st->edges_traversed = E * (uint64_t)(hc.iter + 2);
        st->edges_relaxed = st->edges_traversed;
        st->residual = hc.residual;
        st->device_ms = ms;
    }
    return OLV_OK;
}

extern "C" int olv_wpr_ctx_destroy(olv_wpr_ctx *c) {
    if (!c) return OLV_OK;
    c->fwd.destroy();
    c->bwd.destroy();
    c->W.release(); c->r.release(); c->s2.release(); c->tp.release(); c->lam2.release();
    c->t.release(); c->gbuf.release(); c->ctl.release();
    delete c;
    return OLV_OK;
}
