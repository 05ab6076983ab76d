// Deterministic segmented row sums over a CSR-shaped structure (row
// offsets `ptr`, neighbour ids `idx`), the shared core of PageRank, weighted
// PageRank and its adjoint.
//
// Rows are cut into row blocks (RowPlan): consecutive rows holding at most
// kNnz entries and kRows rows, or one row longer than kNnz.  For a short-row
// block the CTA stages every term of the block in shared memory, then sums
// each row in entry order with compensated (two-sum) FP32 arithmetic: rows
// of at most kShort entries by one thread, longer ones by a warp with a
// fixed-shape tree.  A long row is cut into kSeg-entry segments summed by
// k_row_segments (one CTA each, fixed tree) and folded in segment order.
// Every sum thus has a fixed evaluation order: results do not depend on
// scheduling, and each carries about one FP32 rounding.
//
// An Op supplies:
//   void begin()                                per-launch setup (ping-pong choice)
//   float term(uint32_t e, uint32_t j)          value of entry e with neighbour j
//   void finish(uint32_t row, float s, float c, double &res, double &aux)
//                                               consume the row sum s + c; res
//                                               and aux are FP64 CTA partials
//   const uint32_t *done                        the kernels return when *done
#pragma once
#include <vector>

#include "olv_internal.cuh"

namespace olv {

constexpr uint32_t kNnz = 2048;      // entries staged per row block
constexpr uint32_t kRows = 256;      // rows per row block at most (one per thread)
constexpr uint32_t kSeg = 4096;      // entries per segment of a long row
constexpr uint32_t kShort = 32;      // rows up to this length are summed by one thread
constexpr int kGather = kNnz / kBlock;

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

struct RowPlan {
    DevBuf blocks, segbase, seg_range, seg_row, segs, partials;
    uint32_t nblocks = 0, nsegs = 0;
    void release() {
        blocks.release(); segbase.release(); seg_range.release(); seg_row.release();
        segs.release(); partials.release();
    }
};

// Build the row blocks of a (device) offset array with n rows.
inline int build_row_plan(const uint32_t *ptr_dev, uint32_t n, cudaStream_t s, RowPlan &p) {
    std::vector<uint32_t> cp((size_t)n + 1);
    OLV_CUDA(cudaMemcpyAsync(cp.data(), ptr_dev, ((size_t)n + 1) * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> b;
    b.reserve(cp[n] / kNnz + n / kRows + 16);
    b.push_back(0);
    uint32_t v = 0;
    while (v < n) {
        const uint32_t start = v;
        if (cp[v + 1] - cp[v] > kNnz) {
            v++;
        } else {
            while (v < n && v - start < kRows && cp[v + 1] - cp[start] <= kNnz) v++;
        }
        b.push_back(v);
    }
    p.nblocks = (uint32_t)b.size() - 1;
    std::vector<uint32_t> segbase(p.nblocks, 0xffffffffu);
    std::vector<uint2> ranges;
    std::vector<uint32_t> segrow;
    for (uint32_t k = 0; k < p.nblocks; k++) {
        const uint32_t e0 = cp[b[k]], e1 = cp[b[k + 1]];
        if (e1 - e0 <= kNnz) continue;
        segbase[k] = (uint32_t)ranges.size();
        for (uint32_t x = e0; x < e1; x += kSeg) {
            ranges.push_back(make_uint2(x, e1 - x > kSeg ? x + kSeg : e1));
            segrow.push_back(b[k]);
        }
    }
    p.nsegs = (uint32_t)ranges.size();
    OLV_TRY(p.blocks.ensure(b.size() * 4));
    OLV_TRY(p.segbase.ensure(segbase.size() * 4 + 16));
    OLV_TRY(p.seg_range.ensure(ranges.size() * 8 + 16));
    OLV_TRY(p.segs.ensure(ranges.size() * 8 + 16));
    OLV_TRY(p.seg_row.ensure(segrow.size() * 4 + 16));
    OLV_TRY(p.partials.ensure((size_t)p.nblocks * 16 + 16));
    OLV_CUDA(cudaMemcpyAsync(p.blocks.p, b.data(), b.size() * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(p.segbase.p, segbase.data(), segbase.size() * 4,
                             cudaMemcpyHostToDevice, s));
    if (!ranges.empty()) {
        OLV_CUDA(cudaMemcpyAsync(p.seg_range.p, ranges.data(), ranges.size() * 8,
                                 cudaMemcpyHostToDevice, s));
        OLV_CUDA(cudaMemcpyAsync(p.seg_row.p, segrow.data(), segrow.size() * 4,
                                 cudaMemcpyHostToDevice, s));
    }
    OLV_CUDA(cudaStreamSynchronize(s));
    return OLV_OK;
}

template <class Op>
__global__ void __launch_bounds__(kBlock)
k_row_segments(const uint32_t *__restrict__ idx, const uint2 *__restrict__ seg_range, Op op,
               float2 *__restrict__ segs) {
    if (*op.done) return;
    op.begin();
    const uint2 r = seg_range[blockIdx.x];
    __shared__ float s_red[2][kBlock];
    constexpr int U = kSeg / kBlock;
    uint32_t j[U];
#pragma unroll
    for (int q = 0; q < U; q++) {
        const uint32_t i = r.x + threadIdx.x + q * kBlock;
        j[q] = i < r.y ? __ldg(&idx[i]) : 0xffffffffu;
    }
    float x[U];
#pragma unroll
    for (int q = 0; q < U; q++) {
        const uint32_t i = r.x + threadIdx.x + q * kBlock;
        x[q] = j[q] != 0xffffffffu ? op.term(i, j[q]) : 0.0f;
    }
    float s = 0.0f, c = 0.0f;
#pragma unroll
    for (int q = 0; q < U; q++) two_sum_acc(s, c, x[q]);
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

template <class Op>
__global__ void __launch_bounds__(kBlock, 8)
k_row_blocks(const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ idx,
             const uint32_t *__restrict__ blocks, const uint32_t *__restrict__ segbase,
             const float2 *__restrict__ segs, Op op, double *__restrict__ partials) {
    if (*op.done) return;
    op.begin();
    const uint32_t r0 = blocks[blockIdx.x], r1 = blocks[blockIdx.x + 1];
    const uint32_t e0 = ptr[r0], e1 = ptr[r1];
    __shared__ float s_val[kNnz];
    __shared__ double s_dred[2][kBlock / 32];
    __shared__ uint32_t s_long[kNnz / (kShort + 1) + 1];
    __shared__ uint32_t s_nlong;
    if (threadIdx.x == 0) s_nlong = 0;
    double res = 0.0, aux = 0.0;
    if (e1 - e0 <= kNnz) {
        const uint32_t n = e1 - e0;
        uint32_t j[kGather];
#pragma unroll
        for (int q = 0; q < kGather; q++) {
            const uint32_t i = threadIdx.x + q * kBlock;
            j[q] = i < n ? __ldg(&idx[e0 + i]) : 0u;
        }
#pragma unroll
        for (int q = 0; q < kGather; q++) {
            const uint32_t i = threadIdx.x + q * kBlock;
            if (i < n) s_val[i] = op.term(e0 + i, j[q]);
        }
        __syncthreads();
        for (uint32_t v = r0 + threadIdx.x; v < r1; v += kBlock) {
            const uint32_t b = ptr[v] - e0, e = ptr[v + 1] - e0;
            if (e - b > kShort) {
                s_long[atomicAdd(&s_nlong, 1u)] = v;
                continue;
            }
            float s = 0.0f, c = 0.0f;
            for (uint32_t i = b; i < e; i++) two_sum_acc(s, c, s_val[i]);
            op.finish(v, s, c, res, aux);
        }
        __syncthreads();
        const uint32_t nlong = s_nlong, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (uint32_t k = wid; k < nlong; k += kBlock / 32) {
            const uint32_t v = s_long[k];
            const uint32_t b = ptr[v] - e0, e = ptr[v + 1] - e0;
            float s = 0.0f, c = 0.0f;
            for (uint32_t i = b + lane; i < e; i += 32) two_sum_acc(s, c, s_val[i]);
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const float s2 = __shfl_down_sync(0xffffffffu, s, o);
                const float c2 = __shfl_down_sync(0xffffffffu, c, o);
                pair_add(s, c, s2, c2);
            }
            if (lane == 0) op.finish(v, s, c, res, aux);
        }
    } else if (threadIdx.x == 0) {
        const uint32_t first = segbase[blockIdx.x];
        const uint32_t nseg = (e1 - e0 + kSeg - 1) / kSeg;
        float s = 0.0f, c = 0.0f;
        for (uint32_t k = 0; k < nseg; k++) {
            const float2 p = segs[first + k];
            pair_add(s, c, p.x, p.y);
        }
        op.finish(r0, s, c, res, aux);
    }
    // fixed-order CTA reduction of the FP64 partials
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        res += __shfl_down_sync(0xffffffffu, res, o);
        aux += __shfl_down_sync(0xffffffffu, aux, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_dred[0][threadIdx.x >> 5] = res;
        s_dred[1][threadIdx.x >> 5] = aux;
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

// Add the kernels of one row pass (segments, then blocks) to a launch sink.
template <class Op, class Sink>
int row_pass(const RowPlan &p, const uint32_t *ptr, const uint32_t *idx, Op &op, Sink &&sink) {
    const uint32_t *blocks = p.blocks.as<uint32_t>();
    const uint32_t *segbase = p.segbase.as<uint32_t>();
    const uint2 *seg_range = p.seg_range.as<uint2>();
    float2 *segs = p.segs.as<float2>();
    const float2 *csegs = segs;
    double *partials = p.partials.as<double>();
    if (p.nsegs) {
        void *a_seg[] = {&idx, &seg_range, &op, &segs};
        OLV_TRY(sink((const void *)k_row_segments<Op>, dim3(p.nsegs), dim3(kBlock), a_seg));
    }
    void *a_blk[] = {&ptr, &idx, &blocks, &segbase, &csegs, &op, &partials};
    OLV_TRY(sink((const void *)k_row_blocks<Op>, dim3(p.nblocks), dim3(kBlock), a_blk));
    return OLV_OK;
}

// Fixed-order fold of the per-CTA FP64 partials of a row pass into an
// iteration control block; decides convergence and sets the graph loop
// condition.  partials[2i] are |x' - x| sums.
struct IterCtl {
    double residual;
    double aux;
    double tol;
    uint32_t iter;
    uint32_t done;
    uint32_t max_it;
    uint32_t pad;
};

constexpr int kFoldThreads = 1024;

static __global__ void __launch_bounds__(kFoldThreads)
k_iter_fold(IterCtl *ctl, const double *__restrict__ partials, uint32_t nparts,
            cudaGraphConditionalHandle h, int use_cond) {
    __shared__ double s[2][kFoldThreads];
    if (ctl->done) {
        if (use_cond && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
        return;
    }
    double a = 0, b = 0;
    for (uint32_t i = threadIdx.x; i < nparts; i += kFoldThreads) {
        a += partials[2 * i];
        b += partials[2 * i + 1];
    }
    s[0][threadIdx.x] = a;
    s[1][threadIdx.x] = b;
    __syncthreads();
    for (int w = kFoldThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < (uint32_t)w) {
            s[0][threadIdx.x] += s[0][threadIdx.x + w];
            s[1][threadIdx.x] += s[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ctl->residual = s[0][0];
        ctl->aux = s[1][0];
        ctl->iter++;
        if (ctl->residual < ctl->tol || ctl->iter >= ctl->max_it) ctl->done = 1;
        if (use_cond) cudaGraphSetConditional(h, ctl->done ? 0u : 1u);
    }
}

}  // namespace olv
