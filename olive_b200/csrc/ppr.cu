// K personalised PageRank vectors on a general graph, advanced together as a
// sparse x dense-K product (no reference counterpart; each vector follows
// PageRank.cu:51-75 with the teleport to its own seed).
//
// Result contract, per vector k with seed s_k (K <= 32), from r_k = e_{s_k}:
//   r_k'[v] = alpha * (sum_{u->v} r_k[u] / outdeg(u)) + [v == s_k] * ((1-alpha) + alpha * d_k)
// with d_k the dangling mass of r_k (it returns to the seed); stop after max_it
// iterations or when max_k sum_v |r_k' - r_k| < tol.  FP32 values, FP64
// residual and dangling sums.
//
// Layout: the reverse graph relabelled by in-degree (longest rows first,
// olv_rowtiles.cuh's plan), one 128-byte row of 32 floats per vertex for the
// values x and for the scaled contributions y = x / outdeg (ping-pong).
// Each iteration is one pull: a group of 8 lanes per row, each lane holding
// four vectors (a float4), walks the row's in-edges in order, gathers the
// 128-byte contribution row of every in-neighbour and adds it with
// compensated (two-sum) FP32 arithmetic, so the sums have a fixed order and
// about one rounding each.  Rows longer than kPprLong are summed in fixed
// kPprSeg-edge segments first and the segments folded in order.  The same
// pass writes x', y' and per-CTA FP64 partials of |x' - x| and of the new
// dangling mass; a one-CTA kernel folds the partials in a fixed order and
// decides convergence on the device, inside a CUDA graph.
#include <algorithm>
#include <vector>

#include "olive_b200/olv_advance.cuh"
#include "olv_graphexec.cuh"
#include "olv_internal.cuh"
#include "olv_rowtiles.cuh"

namespace olv {

constexpr int kPprK = 32;                // vectors per row (K is padded to 32)
constexpr uint32_t kPprLong = 1024;      // rows with more in-edges are segmented
constexpr uint32_t kPprSeg = 1024;       // in-edges per segment
constexpr int kPprMinBlocks = 4;
constexpr uint32_t kPprCTAs = 148 * kPprMinBlocks;   // fixed grid: fixed partial order

struct PprCtl {
    double res[kPprK];      // residual of the last completed iteration, per vector
    double dang[kPprK];     // dangling mass of the current iterate, per vector
    uint32_t seed[kPprK];   // seeds in the relabelled ids (0xffffffff: padding)
    double alpha;
    double tol;
    double max_res;
    uint32_t iter;
    uint32_t max_it;
    uint32_t done;
};

// Compensated accumulation of four lanes' values (Knuth's two-sum).
struct Acc4 {
    float4 s, c;
    __device__ __forceinline__ void zero() {
        s = make_float4(0, 0, 0, 0);
        c = s;
    }
    __device__ __forceinline__ static void add1(float &s, float &c, float x) {
        const float t = s + x;
        const float bp = t - s;
        c += (s - (t - bp)) + (x - bp);
        s = t;
    }
    __device__ __forceinline__ void add(float4 x) {
        add1(s.x, c.x, x.x);
        add1(s.y, c.y, x.y);
        add1(s.z, c.z, x.z);
        add1(s.w, c.w, x.w);
    }
    __device__ __forceinline__ void add_pair(float4 xs, float4 xc) {
        add(xs);
        c.x += xc.x;
        c.y += xc.y;
        c.z += xc.z;
        c.w += xc.w;
    }
    __device__ __forceinline__ float4 value() const {
        return make_float4(s.x + c.x, s.y + c.y, s.z + c.z, s.w + c.w);
    }
};

// Sum of y rows over in-edges [b, e) of one row by an 8-lane group: lane q of
// the group holds vectors 4q..4q+3; the group reads 8 in-neighbour ids at a
// time (one per lane) and broadcasts them.
__device__ __forceinline__ void ppr_row_sum(const uint32_t *__restrict__ idx,
                                            const float4 *__restrict__ y, uint32_t b, uint32_t e,
                                            uint32_t q, unsigned gmask, int gbase, Acc4 &acc) {
    for (uint32_t base = b; base < e; base += 8) {
        const uint32_t j = base + q;
        const uint32_t u = j < e ? __ldcs(&idx[j]) : 0u;
        const uint32_t n = min(8u, e - base);
#pragma unroll
        for (uint32_t h = 0; h < 8; h += 4) {   // four 16-byte row pieces in flight per lane
            float4 v[4];
#pragma unroll
            for (uint32_t t = 0; t < 4; t++) {
                const uint32_t ut = __shfl_sync(gmask, u, gbase + (int)(h + t));
                v[t] = h + t < n ? __ldg(&y[(size_t)ut * (kPprK / 4) + q])
                                 : make_float4(0, 0, 0, 0);
            }
#pragma unroll
            for (uint32_t t = 0; t < 4; t++)
                if (h + t < n) acc.add(v[t]);
        }
    }
}

// Long rows: segment s of the list sums its in-edges into (sum, comp) rows.
__global__ void __launch_bounds__(kBlock, kPprMinBlocks)
k_ppr_segments(const uint32_t *__restrict__ idx, const uint4 *__restrict__ segs,
               uint32_t nsegs, const PprCtl *ctl, const float4 *__restrict__ y0,
               const float4 *__restrict__ y1, float4 *__restrict__ seg_sum,
               float4 *__restrict__ seg_comp) {
    if (ctl->done) return;
    const float4 *y = (ctl->iter & 1) ? y1 : y0;
    const uint32_t lane = threadIdx.x & 31, g = lane >> 3, q = lane & 7;
    const unsigned gmask = 0xffu << (8 * g);
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t s0 = warp * 4; s0 < nsegs; s0 += nwarps * 4) {
        const uint32_t s = s0 + g;
        Acc4 acc;
        acc.zero();
        if (s < nsegs) {
            const uint4 sg = segs[s];   // (row, begin, end, -)
            ppr_row_sum(idx, y, sg.y, sg.z, q, gmask, (int)(8 * g), acc);
            seg_sum[(size_t)s * 8 + q] = acc.s;
            seg_comp[(size_t)s * 8 + q] = acc.c;
        }
    }
}

// One pull over all rows: sums (or folded segments), the update, the next
// contributions, and per-CTA FP64 partials of |x' - x| and the dangling mass.
__global__ void __launch_bounds__(kBlock, kPprMinBlocks)
k_ppr_rows(const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ idx,
           const uint32_t *__restrict__ outdeg, uint32_t n, uint32_t nlong,
           const uint32_t *__restrict__ seg_first, const float4 *__restrict__ seg_sum,
           const float4 *__restrict__ seg_comp, PprCtl *ctl, float a_hi, float a_lo,
           float4 *__restrict__ x, float4 *__restrict__ y0, float4 *__restrict__ y1,
           double *__restrict__ partials) {
    __shared__ double s_part[kBlock / 32][2 * kPprK];
    if (ctl->done) return;
    const bool odd = ctl->iter & 1;
    const float4 *yin = odd ? y1 : y0;
    float4 *yout = odd ? y0 : y1;
    const uint32_t lane = threadIdx.x & 31, g = lane >> 3, q = lane & 7;
    const unsigned gmask = 0xffu << (8 * g);
    const uint32_t wl = threadIdx.x >> 5;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    // this lane's four seeds and their constant terms ((1-alpha) + alpha d_k)
    uint32_t sd[4];
    float st[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
        sd[t] = ctl->seed[4 * q + t];
        st[t] = (float)((1.0 - ctl->alpha) + ctl->alpha * ctl->dang[4 * q + t]);
    }
    double res[4] = {0, 0, 0, 0}, dang[4] = {0, 0, 0, 0};
    for (uint32_t r0 = warp * 4; r0 < n; r0 += nwarps * 4) {
        const uint32_t r = r0 + g;
        if (r < n) {
            Acc4 acc;
            acc.zero();
            if (r < nlong) {
                for (uint32_t s = seg_first[r]; s < seg_first[r + 1]; s++)
                    acc.add_pair(seg_sum[(size_t)s * 8 + q], seg_comp[(size_t)s * 8 + q]);
            } else {
                ppr_row_sum(idx, yin, __ldg(&ptr[r]), __ldg(&ptr[r + 1]), q, gmask, (int)(8 * g),
                            acc);
            }
            const float4 sv = acc.value();
            const float4 old = x[(size_t)r * 8 + q];
            const float sum[4] = {sv.x, sv.y, sv.z, sv.w};
            const float ov[4] = {old.x, old.y, old.z, old.w};
            float nv[4];
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const float base = sd[t] == r ? st[t] : 0.0f;
                nv[t] = fmaf(a_hi, sum[t], fmaf(a_lo, sum[t], base));
                res[t] += fabs((double)nv[t] - (double)ov[t]);
            }
            const float4 nx = make_float4(nv[0], nv[1], nv[2], nv[3]);
            x[(size_t)r * 8 + q] = nx;
            const uint32_t d = __ldg(&outdeg[r]);
            if (d) {
                const float fd = (float)d;
                yout[(size_t)r * 8 + q] = make_float4(__fdiv_rn(nv[0], fd), __fdiv_rn(nv[1], fd),
                                                      __fdiv_rn(nv[2], fd), __fdiv_rn(nv[3], fd));
            } else {
                yout[(size_t)r * 8 + q] = make_float4(0, 0, 0, 0);
#pragma unroll
                for (int t = 0; t < 4; t++) dang[t] += (double)nv[t];
            }
        }
    }
    // fixed-order reduction: the warp's four groups, then the CTA's warps
#pragma unroll
    for (int t = 0; t < 4; t++) {
        res[t] += __shfl_xor_sync(0xffffffffu, res[t], 8);
        res[t] += __shfl_xor_sync(0xffffffffu, res[t], 16);
        dang[t] += __shfl_xor_sync(0xffffffffu, dang[t], 8);
        dang[t] += __shfl_xor_sync(0xffffffffu, dang[t], 16);
    }
    if (g == 0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            s_part[wl][4 * q + t] = res[t];
            s_part[wl][kPprK + 4 * q + t] = dang[t];
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * kPprK) {
        double a = 0;
        for (int w = 0; w < kBlock / 32; w++) a += s_part[w][threadIdx.x];
        partials[(size_t)blockIdx.x * 2 * kPprK + threadIdx.x] = a;
    }
}

// Fold the per-CTA partials in a fixed order, publish residuals and dangling
// masses, decide convergence.
__global__ void k_ppr_reduce(PprCtl *ctl, const double *__restrict__ partials, uint32_t nparts,
                             cudaGraphConditionalHandle h, int use_cond) {
    if (ctl->done) {
        if (use_cond && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
        return;
    }
    const uint32_t k = threadIdx.x;   // 2 * kPprK threads
    double a = 0;
    for (uint32_t i = 0; i < nparts; i++) a += partials[(size_t)i * 2 * kPprK + k];
    __syncthreads();
    if (k < kPprK)
        ctl->res[k] = a;
    else
        ctl->dang[k - kPprK] = a;
    __syncthreads();
    if (k == 0) {
        double m = 0;
        for (int t = 0; t < kPprK; t++) m = ctl->res[t] > m ? ctl->res[t] : m;
        ctl->max_res = m;
        ctl->iter++;
        if (m < ctl->tol || ctl->iter >= ctl->max_it) ctl->done = 1;
        if (use_cond) cudaGraphSetConditional(h, ctl->done ? 0u : 1u);
    }
}

// Start state: x = e_{s_k}, y = x / outdeg, d_k = [outdeg(s_k) == 0].
__global__ void k_ppr_init_seeds(PprCtl *ctl, const uint32_t *__restrict__ outdeg, float *x,
                                 float *y0, double alpha, double tol, uint32_t max_it) {
    const int k = threadIdx.x;   // kPprK threads
    const uint32_t s = ctl->seed[k];
    if (s != 0xffffffffu) {
        const uint32_t d = outdeg[s];
        x[(size_t)s * kPprK + k] = 1.0f;
        y0[(size_t)s * kPprK + k] = d ? __fdiv_rn(1.0f, (float)d) : 0.0f;
        ctl->dang[k] = d ? 0.0 : 1.0;
    } else {
        ctl->dang[k] = 0.0;
    }
    ctl->res[k] = 0.0;
    if (k == 0) {
        ctl->alpha = alpha;
        ctl->tol = tol;
        ctl->max_it = max_it;
        ctl->iter = 0;
        ctl->max_res = 0;
        ctl->done = max_it == 0;
    }
}

__global__ void k_ppr_set_seeds(PprCtl *ctl, const uint32_t *__restrict__ seeds, int K,
                                const uint32_t *__restrict__ newid) {
    const int k = threadIdx.x;
    ctl->seed[k] = k < K ? newid[seeds[k]] : 0xffffffffu;
}

// out[v][k] = x[newid[v]][k] for k < K (the caller's ids and width).
__global__ void k_ppr_unpermute(const float *__restrict__ x, const uint32_t *__restrict__ newid,
                                uint32_t V, int K, float *__restrict__ out) {
    const uint64_t total = (uint64_t)V * K;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = i / K, k = i - v * K;
        out[i] = x[(size_t)newid[v] * kPprK + k];
    }
}

__global__ void k_outdeg_in_order(const uint32_t *__restrict__ rowptr,
                                  const uint32_t *__restrict__ perm, uint32_t V, uint32_t *d) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = perm[i];
        d[i] = rowptr[v + 1] - rowptr[v];
    }
}

// ------------------------------------------------------------------ host --
struct PprState {
    TilePlan tp;                       // relabelled reverse graph (rows by in-degree)
    DevBuf outdeg, x, y, ctl, partials, segs, seg_first, seg_sum, seg_comp, seeds, out;
    uint32_t nlong = 0, nsegs = 0;
    WhileGraph graph;
    float a_hi = 0, a_lo = 0;
    ~PprState() {
        graph.destroy();
        tp.release(); outdeg.release(); x.release(); y.release(); ctl.release();
        partials.release(); segs.release(); seg_first.release(); seg_sum.release();
        seg_comp.release(); seeds.release(); out.release();
    }
};

static int build_ppr_state(olv_graph *g, PprState &p) {
    const uint32_t V = g->V;
    cudaStream_t s = g->stream;
    OLV_TRY(build_tile_plan(g->colptr.as<uint32_t>(), g->rowidx.as<uint32_t>(), V, s, p.tp));
    OLV_TRY(p.outdeg.ensure((size_t)V * 4 + 16));
    k_outdeg_in_order<<<g->num_sms * 8, kBlock, 0, s>>>(
        g->rowptr.as<uint32_t>(), p.tp.perm.as<uint32_t>(), V, p.outdeg.as<uint32_t>());
    // long rows are a prefix of the in-degree order: their segments
    std::vector<uint32_t> ptr((size_t)V + 1);
    OLV_CUDA(cudaMemcpyAsync(ptr.data(), p.tp.ptr.p, ((size_t)V + 1) * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    uint32_t nlong = 0;
    while (nlong < V && ptr[nlong + 1] - ptr[nlong] > kPprLong) nlong++;
    std::vector<uint4> segs;
    std::vector<uint32_t> first((size_t)nlong + 1, 0);
    for (uint32_t r = 0; r < nlong; r++) {
        first[r] = (uint32_t)segs.size();
        for (uint32_t b = ptr[r]; b < ptr[r + 1]; b += kPprSeg)
            segs.push_back(make_uint4(r, b, std::min(ptr[r + 1], b + kPprSeg), 0));
    }
    first[nlong] = (uint32_t)segs.size();
    p.nlong = nlong;
    p.nsegs = (uint32_t)segs.size();
    const size_t rows = (size_t)V * kPprK * 4;
    OLV_TRY(p.x.ensure(rows + 64));
    OLV_TRY(p.y.ensure(2 * rows + 64));
    OLV_TRY(p.ctl.ensure(sizeof(PprCtl)));
    OLV_TRY(p.partials.ensure((size_t)kPprCTAs * 2 * kPprK * 8));
    OLV_TRY(p.segs.ensure(segs.size() * 16 + 16));
    OLV_TRY(p.seg_first.ensure(first.size() * 4 + 16));
    OLV_TRY(p.seg_sum.ensure(segs.size() * kPprK * 4 + 16));
    OLV_TRY(p.seg_comp.ensure(segs.size() * kPprK * 4 + 16));
    OLV_TRY(p.seeds.ensure(kPprK * 4));
    if (!segs.empty())
        OLV_CUDA(cudaMemcpyAsync(p.segs.p, segs.data(), segs.size() * 16, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(p.seg_first.p, first.data(), first.size() * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaStreamSynchronize(s));   // the host vectors die here
    return OLV_OK;
}

template <class Sink>
static int ppr_iteration(olv_graph *g, PprState &p, Sink &&sink, cudaGraphConditionalHandle h,
                         int use_cond) {
    PprCtl *ctl = p.ctl.as<PprCtl>();
    const uint32_t *idx = p.tp.idx.as<uint32_t>(), *ptr = p.tp.ptr.as<uint32_t>();
    const uint32_t *outdeg = p.outdeg.as<uint32_t>();
    const uint32_t *seg_first = p.seg_first.as<uint32_t>();
    const uint4 *segs = p.segs.as<uint4>();
    float4 *x = p.x.as<float4>();
    float4 *y0 = p.y.as<float4>();
    float4 *y1 = y0 + (size_t)g->V * (kPprK / 4);
    float4 *seg_sum = p.seg_sum.as<float4>(), *seg_comp = p.seg_comp.as<float4>();
    double *partials = p.partials.as<double>();
    uint32_t n = g->V, nlong = p.nlong, nsegs = p.nsegs, nparts = kPprCTAs;
    float a_hi = p.a_hi, a_lo = p.a_lo;
    if (nsegs) {
        void *a_seg[] = {&idx, &segs, &nsegs, &ctl, &y0, &y1, &seg_sum, &seg_comp};
        OLV_TRY(sink((const void *)k_ppr_segments, dim3(kPprCTAs), dim3(kBlock), a_seg));
    }
    void *a_rows[] = {&ptr, &idx, &outdeg, &n, &nlong, &seg_first, &seg_sum, &seg_comp,
                      &ctl, &a_hi, &a_lo, &x, &y0, &y1, &partials};
    OLV_TRY(sink((const void *)k_ppr_rows, dim3(kPprCTAs), dim3(kBlock), a_rows));
    void *a_red[] = {&ctl, &partials, &nparts, &h, &use_cond};
    OLV_TRY(sink((const void *)k_ppr_reduce, dim3(1), dim3(2 * kPprK), a_red));
    return OLV_OK;
}

}  // namespace olv

using namespace olv;

static PprState *ppr_state(olv_graph *g) { return static_cast<PprState *>(g->ppr_state); }

void olv::release_ppr_state(olv_graph *g) {
    delete ppr_state(g);
    g->ppr_state = nullptr;
}

extern "C" int olv_ppr_batch(olv_graph *g, const uint32_t *seeds, int K, double alpha,
                             int max_it, double tol, float *out, olv_stats *st) {
    OLV_CHECK_ARG(g && seeds && out, "olv_ppr_batch: null pointer");
    OLV_CHECK_ARG(K >= 1 && K <= kPprK, "olv_ppr_batch: K must be in [1, %d]", kPprK);
    OLV_CHECK_ARG(alpha >= 0.0 && alpha < 1.0, "olv_ppr_batch: alpha must be in [0,1)");
    OLV_CHECK_ARG(max_it >= 0, "olv_ppr_batch: max_it must be >= 0");
    OLV_CHECK_ARG(g->V > 0, "olv_ppr_batch: empty graph");
    cudaStream_t s = g->stream;
    const bool dev_seeds = is_device_ptr(seeds);
    std::vector<uint32_t> hs(K);
    if (dev_seeds) {
        OLV_CUDA(cudaMemcpyAsync(hs.data(), seeds, (size_t)K * 4, cudaMemcpyDeviceToHost, s));
        OLV_CUDA(cudaStreamSynchronize(s));
    } else {
        std::copy(seeds, seeds + K, hs.begin());
    }
    for (int k = 0; k < K; k++)
        OLV_CHECK_ARG(hs[k] < g->V, "olv_ppr_batch: seed %u out of range (V=%u)", hs[k], g->V);
    PprState *ps = ppr_state(g);
    if (!ps) {
        ps = new PprState();
        g->ppr_state = ps;
        int r = build_ppr_state(g, *ps);
        if (r != OLV_OK) {
            release_ppr_state(g);
            return r;
        }
    }
    PprState &p = *ps;
    p.a_hi = (float)alpha;
    p.a_lo = (float)(alpha - (double)p.a_hi);
    const size_t rows = (size_t)g->V * kPprK * 4;
    const bool dev_out = is_device_ptr(out);
    if (!dev_out) OLV_TRY(p.out.ensure((size_t)g->V * K * 4 + 16));
    float *dst = dev_out ? out : p.out.as<float>();
    OLV_CUDA(cudaEventRecord(g->ev0, s));
    OLV_CUDA(cudaMemcpyAsync(p.seeds.p, hs.data(), (size_t)K * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemsetAsync(p.x.p, 0, rows, s));
    OLV_CUDA(cudaMemsetAsync(p.y.p, 0, rows, s));   // y0; y1 is written before it is read
    k_ppr_set_seeds<<<1, kPprK, 0, s>>>(p.ctl.as<PprCtl>(), p.seeds.as<uint32_t>(), K,
                                        p.tp.newid.as<uint32_t>());
    k_ppr_init_seeds<<<1, kPprK, 0, s>>>(p.ctl.as<PprCtl>(), p.outdeg.as<uint32_t>(),
                                         p.x.as<float>(), p.y.as<float>(), alpha, tol,
                                         (uint32_t)max_it);
    OLV_CUDA(cudaGetLastError());
    bool launched = false;
    if (g->tune.use_graphs && max_it > 0) {
        if (!p.graph.ready) {
            int r = p.graph.begin();
            auto sink = [&](const void *f, dim3 gr, dim3 bl, void **args) {
                return p.graph.add(f, gr, bl, args);
            };
            if (r == OLV_OK) r = ppr_iteration(g, p, sink, p.graph.handle, 1);
            if (r == OLV_OK) r = p.graph.finish();
            if (r != OLV_OK) p.graph.destroy();
        }
        if (p.graph.ready) {
            OLV_TRY(p.graph.launch(s));
            launched = true;
        }
    }
    if (!launched) {
        auto launch = [&](const void *f, dim3 gr, dim3 bl, void **args) {
            OLV_CUDA(cudaLaunchKernel(f, gr, bl, args, 0, s));
            return OLV_OK;
        };
        for (int it = 0; it < max_it; it++) OLV_TRY(ppr_iteration(g, p, launch, 0, 0));
    }
    k_ppr_unpermute<<<g->num_sms * 8, kBlock, 0, s>>>(p.x.as<float>(), p.tp.newid.as<uint32_t>(),
                                                     g->V, K, dst);
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaEventRecord(g->ev1, s));
    PprCtl hc;
    OLV_CUDA(cudaMemcpyAsync(&hc, p.ctl.p, sizeof hc, cudaMemcpyDeviceToHost, s));
    if (!dev_out)
        OLV_CUDA(cudaMemcpyAsync(out, dst, (size_t)g->V * K * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    if (st) {
        float ms = 0;
        OLV_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        st->iterations = hc.iter;
        st->pull_steps = 0;
        st->vertices_reached = g->V;
        st->edges_traversed = g->E * (uint64_t)hc.iter;
        st->edges_relaxed = g->E * (uint64_t)hc.iter * (uint64_t)K;
        st->residual = hc.max_res;
        st->device_ms = ms;
    }
    return OLV_OK;
}
