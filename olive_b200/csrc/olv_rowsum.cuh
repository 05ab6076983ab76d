// Deterministic segmented row sums over a CSR-shaped structure (row
// offsets `ptr`, neighbour ids `idx`), the shared core of PageRank, weighted
// PageRank and its adjoint.
//
// Rows are cut into warp blocks (RowPlan): consecutive rows holding at most
// kNnz entries and kRows rows, or one row longer than kNnz.  A warp reads its
// block's entries in 32-entry strips (kStrips strips of loads in flight) and
// sums them by row with a segmented scan across the lanes (shuffles, a fixed
// shape set by the row offsets), carrying a row that crosses a strip into the
// next strip; all sums use compensated (two-sum) FP32 arithmetic.  A long row
// is cut into kSeg-entry segments summed by k_row_segments (one CTA each,
// fixed tree) and folded in segment order.  Warps take blocks by a fixed
// stride over a fixed grid (kRowCTAs CTAs), so every sum, and every FP64
// partial the row updates produce, has a fixed evaluation order: results do
// not depend on scheduling, and each row sum carries about one FP32 rounding.
//
// An Op supplies:
//   void begin()                                per-launch setup (ping-pong choice)
//   float term(uint32_t e, uint32_t j)          value of entry e with neighbour j
//   struct Row                                  per-row inputs of the update (32-bit words)
//   Row row(uint32_t v)                         load them; a warp loads its block's rows
//                                               together, one coalesced load per lane
//   void finish(uint32_t v, float s, float c, const Row &r, double &res, double &aux)
//                                               consume the row sum s + c; res and aux
//                                               are FP64 partials
//   const uint32_t *done                        the kernels return when *done
#pragma once
#include <vector>

#include "olv_internal.cuh"

namespace olv {

constexpr uint32_t kNnz = 1024;      // entries of a warp block; longer rows are segmented
constexpr uint32_t kRows = 32;       // rows per warp block at most (one per lane)
constexpr uint32_t kSeg = 1024;      // entries per segment of a long row (one warp)
#ifndef OLV_STRIPS
#define OLV_STRIPS 8
#endif
#ifndef OLV_LANE
#define OLV_LANE 4
#endif
constexpr int kStrips = OLV_STRIPS;  // 32-entry strips per warp with loads in flight (segments)
constexpr int kLane = OLV_LANE;      // consecutive entries per lane per round (row blocks)
static_assert(kLane % 4 == 0, "lane entries are read as float4");
constexpr uint32_t kRowCTAs = 148 * 6;   // fixed grid of the row pass (fixed partial order);
                                         // one wave on 148 SMs at 6 CTAs per SM

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
    uint32_t nparts = kRowCTAs;   // FP64 partial pairs one row pass writes
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
    OLV_TRY(p.partials.ensure((size_t)kRowCTAs * 16 + 16));
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

// One warp per segment of a long row: each lane sums its entries (stride 32,
// kStrips loads in flight) in order, then a fixed shuffle tree combines the
// lanes.
template <class Op>
__global__ void __launch_bounds__(kBlock)
k_row_segments(const uint32_t *__restrict__ idx, const uint2 *__restrict__ seg_range,
               uint32_t nsegs, Op op, float2 *__restrict__ segs) {
    if (*op.done) return;
    op.begin();
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t w = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    if (w >= nsegs) return;   // whole warps only
    const uint2 r = seg_range[w];
    float s = 0.0f, c = 0.0f;
    for (uint32_t base = r.x; base < r.y; base += 32 * kStrips) {
        uint32_t j[kStrips];
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            const uint32_t i = base + q * 32 + lane;
            j[q] = i < r.y ? __ldg(&idx[i]) : 0u;
        }
        float x[kStrips];
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            const uint32_t i = base + q * 32 + lane;
            x[q] = i < r.y ? op.term(i, j[q]) : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < kStrips; q++) two_sum_acc(s, c, x[q]);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float s2 = __shfl_down_sync(0xffffffffu, s, o);
        const float c2 = __shfl_down_sync(0xffffffffu, c, o);
        pair_add(s, c, s2, c2);
    }
    if (lane == 0) segs[w] = make_float2(s, c);
}

template <class Op>
__global__ void __launch_bounds__(kBlock, 6)
k_row_warps(const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ idx,
            const uint32_t *__restrict__ blocks, uint32_t nblocks,
            const uint32_t *__restrict__ segbase, const float2 *__restrict__ segs, Op op,
            double *__restrict__ partials) {
    if (*op.done) return;
    op.begin();
    constexpr unsigned kFull = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * kBlock) >> 5;
    double res = 0.0, aux = 0.0;
    const uint32_t wl = threadIdx.x >> 5;
    __shared__ float2 s_sum[kBlock / 32][kRows];        // row sums of the warp's block
    __shared__ uint32_t s_start[kBlock / 32][kRows + 1]; // row starts, then e1
    __shared__ float4 s_x[kBlock / 32][32 * kLane / 4]; // one round of terms, lane-major
    float2 *sum = s_sum[wl];
    uint32_t *start = s_start[wl];
    float *sxf = reinterpret_cast<float *>(s_x[wl]);
    for (uint32_t k = gw; k < nblocks; k += nw) {
        const uint32_t r0 = __ldg(&blocks[k]), r1 = __ldg(&blocks[k + 1]);
        const uint32_t nr = r1 - r0;
        const uint32_t e1 = __ldg(&ptr[r1]);
        // lane i holds the first entry of row r0 + i (all ones past the block)
        const uint32_t pl = lane < nr ? __ldg(&ptr[r0 + lane]) : 0xffffffffu;
        const uint32_t e0 = __shfl_sync(kFull, pl, 0);
        typename Op::Row rd{};   // per-row inputs of row r0 + lane, loaded up front
        if (lane < nr) rd = op.row(r0 + lane);
        if (e1 - e0 > kNnz) {   // one long row: fold its segment sums in order
            if (lane == 0) {
                const uint32_t first = segbase[k];
                const uint32_t nseg = (e1 - e0 + kSeg - 1) / kSeg;
                float s = 0.0f, c = 0.0f;
                for (uint32_t q = 0; q < nseg; q++) {
                    const float2 p = segs[first + q];
                    pair_add(s, c, p.x, p.y);
                }
                op.finish(r0, s, c, rd, res, aux);
            }
            continue;
        }
        start[lane] = lane < nr ? pl : e1;
        if (lane == 0) start[kRows] = e1;
        sum[lane] = make_float2(0.0f, 0.0f);   // empty rows keep 0
        float cs = 0.0f, cc = 0.0f;     // sum of the row carried into the next round
        uint32_t crow = 0xffffffffu;    // that row (block-relative), or none
        for (uint32_t base = e0; base < e1; base += 32 * kLane) {
            // terms of entries base .. base + 32*kLane - 1, coalesced loads
            float x[kLane];
            {
                uint32_t j[kLane];
#pragma unroll
                for (int q = 0; q < kLane; q++) {
                    const uint32_t e = base + q * 32 + lane;
                    j[q] = e < e1 ? __ldg(&idx[e]) : 0u;
                }
#pragma unroll
                for (int q = 0; q < kLane; q++) {
                    const uint32_t e = base + q * 32 + lane;
                    x[q] = e < e1 ? op.term(e, j[q]) : 0.0f;
                }
            }
            __syncwarp();   // the previous round's reads are done
#pragma unroll
            for (int q = 0; q < kLane; q++) sxf[q * 32 + lane] = x[q];
            __syncwarp();
            // this lane's entries: a .. a + kLane - 1, in order
            float xv[kLane];
#pragma unroll
            for (int q = 0; q < kLane / 4; q++) {
                const float4 t4 = s_x[wl][lane * (kLane / 4) + q];
                xv[4 * q] = t4.x;
                xv[4 * q + 1] = t4.y;
                xv[4 * q + 2] = t4.z;
                xv[4 * q + 3] = t4.w;
            }
            const uint32_t a = base + kLane * lane;
            const bool any = a < e1;
            // block-relative row of entry a: the largest k with start(k) <= a
            uint32_t rk = 0;
#pragma unroll
            for (uint32_t step = 16; step; step >>= 1) {
                const uint32_t pk = __shfl_sync(kFull, pl, rk + step);
                if (pk <= a) rk += step;
            }
            // walk the lane's entries: head = part of the first row, rows wholly
            // inside the lane are complete, tail = part of the last row
            uint32_t row = rk, nxt = start[rk + 1];
            float ts = 0.0f, tc = 0.0f, hs = 0.0f, hc = 0.0f;
            bool split = false;
#pragma unroll
            for (int i = 0; i < kLane; i++) {
                const uint32_t e = a + i;
                if (e < e1) {
                    if (e >= nxt) {   // the row ended before e
                        if (!split) {
                            hs = ts;
                            hc = tc;
                            split = true;
                        } else {
                            sum[row] = make_float2(ts, tc);
                        }
                        ts = 0.0f;
                        tc = 0.0f;
                        row++;
                        while (start[row + 1] <= e) row++;   // skip empty rows
                        nxt = start[row + 1];
                    }
                    two_sum_acc(ts, tc, xv[i]);
                }
            }
            // the row carried from the previous round continues in lane 0
            if (lane == 0 && any && rk == crow) {
                if (split)
                    pair_add(hs, hc, cs, cc);
                else
                    pair_add(ts, tc, cs, cc);
            }
            // inclusive segmented scan of the lanes' last-row partials, by row
            const uint32_t key = any ? row : 64u + lane;
            float ss = any ? ts : 0.0f, sc = any ? tc : 0.0f;
#pragma unroll
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const float s2 = __shfl_up_sync(kFull, ss, o);
                const float c2 = __shfl_up_sync(kFull, sc, o);
                const uint32_t k2 = __shfl_up_sync(kFull, key, o);
                if (lane >= o && k2 == key) pair_add(ss, sc, s2, c2);
            }
            // a lane with a row boundary completes its first row with the run
            // of earlier lanes on that row
            const float ps = __shfl_up_sync(kFull, ss, 1);
            const float pc = __shfl_up_sync(kFull, sc, 1);
            const uint32_t pk = __shfl_up_sync(kFull, key, 1);
            if (split) {
                if (lane > 0 && pk == rk) pair_add(hs, hc, ps, pc);
                sum[rk] = make_float2(hs, hc);
            }
            // the lane's last row is complete when it ends within the lane
            const bool ended = any && start[key + 1] <= a + kLane;
            if (ended) sum[key] = make_float2(ss, sc);
            // carry lane 31's last row into the next round unless it ended
            const bool cont = __shfl_sync(kFull, (int)(any && !ended), 31) != 0;
            const float s31 = __shfl_sync(kFull, ss, 31);
            const float c31 = __shfl_sync(kFull, sc, 31);
            const uint32_t k31 = __shfl_sync(kFull, key, 31);
            if (cont) {
                cs = s31;
                cc = c31;
                crow = k31;
            } else {
                crow = 0xffffffffu;
            }
        }
        __syncwarp();
        // every row of the block is updated once, row r0 + lane by lane
        if (lane < nr) {
            const float2 t = sum[lane];
            op.finish(r0 + lane, t.x, t.y, rd, res, aux);
        }
        __syncwarp();
    }
    // fixed-order reduction of the FP64 partials: warp tree, then warps in order
    __shared__ double s_dred[2][kBlock / 32];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        res += __shfl_down_sync(kFull, res, o);
        aux += __shfl_down_sync(kFull, aux, o);
    }
    if (lane == 0) {
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
        uint32_t nsegs = p.nsegs;
        void *a_seg[] = {&idx, &seg_range, &nsegs, &op, &segs};
        OLV_TRY(sink((const void *)k_row_segments<Op>, dim3((nsegs + kBlock / 32 - 1) / (kBlock / 32)),
                     dim3(kBlock), a_seg));
    }
    uint32_t nblocks = p.nblocks;
    void *a_blk[] = {&ptr, &idx, &blocks, &nblocks, &segbase, &csegs, &op, &partials};
    OLV_TRY(sink((const void *)k_row_warps<Op>, dim3(kRowCTAs), dim3(kBlock), a_blk));
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
