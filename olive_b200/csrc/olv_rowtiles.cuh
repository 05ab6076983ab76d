// Row sums over a relabelled, degree-sorted CSR-shaped structure: the pull
// core of PageRank.
//
// The rows (vertices) are renumbered by length, longest first, and the
// neighbour ids inside the rows are renumbered the same way, so that
//   * a warp's rows have nearly equal lengths, and a fixed group of G lanes
//     per row (G = 1..32, chosen from the row length) keeps every lane busy
//     with about kTileU entries per round and no segmented scan;
//   * the high-degree vertices, whose values most rows gather, sit together
//     at the front of every per-vertex array, so their lines stay in L1/L2;
//   * the per-row inputs and outputs are read and written as contiguous runs.
// Rows longer than kTileLong are cut into kTileSeg-entry segments summed by
// k_row_segments (olv_rowsum.cuh) and folded in segment order.
//
// Every sum has a fixed evaluation order: lane j of a row's group adds the
// row's entries j, j+G, j+2G, ... in order with compensated (two-sum) FP32
// arithmetic, then a fixed shuffle tree combines the group's lanes.  Warps
// take tiles by a fixed stride over a fixed grid, so the FP64 partials the
// row updates produce are also summed in a fixed order.
//
// The Op interface is that of olv_rowsum.cuh; row ids are the new ids.
//
// A plan can also keep the neighbour ids (relabel = false): only the rows are
// reordered, `pos` maps each entry to its position in the original structure
// (to permute per-entry values such as edge weights), and PermOp hands the
// original row id to an Op whose per-vertex arrays stay in the original
// order.
#pragma once
#include <algorithm>
#include <vector>

#include "olv_rowsum.cuh"

namespace olv {

constexpr uint32_t kTileLong = 2048;   // rows longer than this are segmented
#ifndef OLV_TILE_SEG
#define OLV_TILE_SEG 512
#endif
constexpr uint32_t kTileSeg = OLV_TILE_SEG;   // entries per segment of a long row
#ifndef OLV_TILE_U
#define OLV_TILE_U 8
#endif
#ifndef OLV_TILE_MINB
#define OLV_TILE_MINB 6
#endif
constexpr int kTileU = OLV_TILE_U;     // entries per lane per round (loads in flight)
constexpr int kTileMinBlocks = OLV_TILE_MINB;   // resident CTAs per SM of the tile pass
constexpr uint32_t kNoSeg = 0xffffffu;
constexpr uint32_t kTileCTAs = 148 * kTileMinBlocks;  // fixed grid of the tile pass
                                                      // (fixed partial order), one wave

// Relabelled structure and its tiles.  tiles[t] = (first row, lg | first
// segment << 8): the tile covers rows first .. first + (32 >> lg) - 1 with
// G = 1 << lg lanes per row; a long row has a tile of its own (lg = 5) whose
// first segment index is below kNoSeg.
struct TilePlan {
    DevBuf perm;      // new id -> old id
    DevBuf newid;     // old id -> new id
    DevBuf ptr;       // [n + 1] row offsets in the new order
    DevBuf idx;       // neighbour (new or original) ids, rows in the new order
    DevBuf pos;       // relabel = false: original position of every entry
    DevBuf tiles, seg_range, segs, partials;
    uint32_t n = 0, ntiles = 0, nsegs = 0;
    void release() {
        perm.release(); newid.release(); ptr.release(); idx.release(); pos.release();
        tiles.release();
        seg_range.release(); segs.release(); partials.release();
    }
};

// idx[ptr[i] + k] = newid[old_idx[old_ptr[perm[i]] + k]] (or the original id
// when newid is null, recording the entry's original position), one warp per
// row.
static __global__ void k_relabel_rows(const uint32_t *__restrict__ old_ptr,
                               const uint32_t *__restrict__ old_idx,
                               const uint32_t *__restrict__ perm, const uint32_t *__restrict__ newid,
                               const uint32_t *__restrict__ ptr, uint32_t n,
                               uint32_t *__restrict__ idx, uint32_t *__restrict__ pos) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w; i < n; i += nw) {
        const uint32_t v = perm[i];
        const uint32_t b = old_ptr[v], e = old_ptr[v + 1], o = ptr[i];
        for (uint32_t k = lane; k < e - b; k += 32) {
            const uint32_t j = old_idx[b + k];
            idx[o + k] = newid ? newid[j] : j;
            if (pos) pos[o + k] = b + k;
        }
    }
}

// out[k] = in[pos[k]]: per-entry values in a plan's entry order.
static __global__ void k_permute_entries(const float *__restrict__ in, const uint32_t *__restrict__ pos,
                                  uint64_t n, float *__restrict__ out) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n;
         k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = in[pos[k]];
}

// An Op over a row-reordered plan (relabel = false): row r of the plan is
// vertex perm[r] of the Op's arrays; entry values come from arrays already
// permuted to the plan's entry order.
template <class Op>
struct PermOp {
    Op op;
    const uint32_t *perm;
    const uint32_t *done;
    __device__ __forceinline__ void begin() { op.begin(); }
    __device__ __forceinline__ float term(uint32_t e, uint32_t j) const { return op.term(e, j); }
    struct Row {
        typename Op::Row r;
        uint32_t v;
    };
    __device__ __forceinline__ Row row(uint32_t r) const {
        const uint32_t v = __ldg(&perm[r]);
        return Row{op.row(v), v};
    }
    __device__ __forceinline__ void finish(uint32_t, float s, float c, const Row &q, double &res,
                                           double &aux) const {
        op.finish(q.v, s, c, q.r, res, aux);
    }
};

// Build the plan from a device row-offset array (n rows) and its neighbour
// array.  The relabelling is a stable counting sort by row length
// (descending), done on the host once per graph.
// lanes_u: entries per lane per round the grouping aims at (rows get the
// fewest lanes G = 1..32 with G * lanes_u >= row length); the autotuner's
// "pr_tile_u".
inline int build_tile_plan(const uint32_t *ptr_dev, const uint32_t *idx_dev, uint32_t n,
                           cudaStream_t s, TilePlan &p, bool relabel = true,
                           uint32_t lanes_u = kTileU) {
    std::vector<uint32_t> cp((size_t)n + 1);
    OLV_CUDA(cudaMemcpyAsync(cp.data(), ptr_dev, ((size_t)n + 1) * 4, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    uint32_t maxd = 0;
    for (uint32_t v = 0; v < n; v++) maxd = std::max(maxd, cp[v + 1] - cp[v]);
    std::vector<uint32_t> start((size_t)maxd + 2, 0);
    for (uint32_t v = 0; v < n; v++) start[maxd - (cp[v + 1] - cp[v]) + 1]++;
    for (size_t d = 1; d < start.size(); d++) start[d] += start[d - 1];
    std::vector<uint32_t> perm(n), newid(n), ptr((size_t)n + 1);
    for (uint32_t v = 0; v < n; v++) {
        const uint32_t i = start[maxd - (cp[v + 1] - cp[v])]++;
        perm[i] = v;
        newid[v] = i;
    }
    ptr[0] = 0;
    for (uint32_t i = 0; i < n; i++) ptr[i + 1] = ptr[i] + (cp[perm[i] + 1] - cp[perm[i]]);
    std::vector<uint2> tiles, ranges;
    for (uint32_t i = 0; i < n;) {
        const uint32_t d = ptr[i + 1] - ptr[i];
        if (d > kTileLong) {
            tiles.push_back(make_uint2(i, 5u | ((uint32_t)ranges.size() << 8)));
            for (uint32_t x = ptr[i]; x < ptr[i + 1]; x += kTileSeg)
                ranges.push_back(make_uint2(x, std::min(ptr[i + 1], x + kTileSeg)));
            i++;
            continue;
        }
        uint32_t lg = 0;
        while (lg < 5 && (1u << lg) * lanes_u < d) lg++;
        tiles.push_back(make_uint2(i, lg | (kNoSeg << 8)));
        i += 32u >> lg;
    }
    if (ranges.size() >= kNoSeg) {
        set_error("row plan: %zu segments exceed the tile format", ranges.size());
        return OLV_ERR_LIMIT;
    }
    p.n = n;
    p.ntiles = (uint32_t)tiles.size();
    p.nsegs = (uint32_t)ranges.size();
    const size_t E = ptr[n];
    OLV_TRY(p.perm.ensure((size_t)n * 4 + 16));
    OLV_TRY(p.newid.ensure((size_t)n * 4 + 16));
    OLV_TRY(p.ptr.ensure(((size_t)n + 1) * 4));
    OLV_TRY(p.idx.ensure(E * 4 + 16));
    if (!relabel) OLV_TRY(p.pos.ensure(E * 4 + 16));
    OLV_TRY(p.tiles.ensure(tiles.size() * 8 + 16));
    OLV_TRY(p.seg_range.ensure(ranges.size() * 8 + 16));
    OLV_TRY(p.segs.ensure(ranges.size() * 8 + 16));
    OLV_TRY(p.partials.ensure((size_t)kTileCTAs * 16 + 16));
    OLV_CUDA(cudaMemcpyAsync(p.perm.p, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(p.newid.p, newid.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(p.ptr.p, ptr.data(), ((size_t)n + 1) * 4, cudaMemcpyHostToDevice, s));
    OLV_CUDA(cudaMemcpyAsync(p.tiles.p, tiles.data(), tiles.size() * 8, cudaMemcpyHostToDevice, s));
    if (!ranges.empty())
        OLV_CUDA(cudaMemcpyAsync(p.seg_range.p, ranges.data(), ranges.size() * 8,
                                 cudaMemcpyHostToDevice, s));
    k_relabel_rows<<<1184, kBlock, 0, s>>>(ptr_dev, idx_dev, p.perm.as<uint32_t>(),
                                          relabel ? p.newid.as<uint32_t>() : nullptr,
                                          p.ptr.as<uint32_t>(), n, p.idx.as<uint32_t>(),
                                          relabel ? nullptr : p.pos.as<uint32_t>());
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaStreamSynchronize(s));
    return OLV_OK;
}

template <class Op>
__global__ void __launch_bounds__(kBlock, kTileMinBlocks)
k_row_tiles(const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ idx,
            const uint2 *__restrict__ tiles, uint32_t ntiles, uint32_t nrows,
            const float2 *__restrict__ segs, Op op, double *__restrict__ partials) {
    if (*op.done) return;
    op.begin();
    constexpr unsigned kFull = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * kBlock + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * kBlock) >> 5;
    double res = 0.0, aux = 0.0;
    uint2 tdn = gw < ntiles ? tiles[gw] : make_uint2(0, 0);
    for (uint32_t t = gw; t < ntiles; t += nw) {
        const uint2 td = tdn;   // the next tile's descriptor is fetched one tile ahead
        if (t + nw < ntiles) tdn = tiles[t + nw];
        const uint32_t lg = td.y & 7u, G = 1u << lg;
        const uint32_t r = td.x + (lane >> lg);
        const uint32_t sub = lane & (G - 1);
        const bool valid = r < nrows;
        uint32_t b = 0, e = 0;
        if (valid) {
            b = __ldg(&ptr[r]);
            e = __ldg(&ptr[r + 1]);
        }
        typename Op::Row rd{};
        if (valid && sub == 0) rd = op.row(r);
        float s = 0.0f, c = 0.0f;
        const uint32_t fs = td.y >> 8;
        if (fs != kNoSeg) {   // one long row: fold its segment sums in order
            if (lane == 0) {
                const uint32_t nseg = (e - b + kTileSeg - 1) / kTileSeg;
                for (uint32_t q = 0; q < nseg; q++) {
                    const float2 pq = segs[fs + q];
                    pair_add(s, c, pq.x, pq.y);
                }
            }
        } else {
            for (uint32_t i = b + sub; i < e; i += G * kTileU) {
                uint32_t j[kTileU];
                float x[kTileU];
#pragma unroll
                for (int u = 0; u < kTileU; u++) {
                    const uint32_t ii = i + u * G;
                    j[u] = ii < e ? __ldg(&idx[ii]) : 0u;
                }
#pragma unroll
                for (int u = 0; u < kTileU; u++) {
                    const uint32_t ii = i + u * G;
                    x[u] = ii < e ? op.term(ii, j[u]) : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < kTileU; u++) two_sum_acc(s, c, x[u]);
            }
            // fixed tree over the row's G lanes (width G keeps groups apart)
            for (uint32_t o = G >> 1; o; o >>= 1) {
                const float s2 = __shfl_down_sync(kFull, s, o, G);
                const float c2 = __shfl_down_sync(kFull, c, o, G);
                pair_add(s, c, s2, c2);
            }
        }
        if (valid && sub == 0) op.finish(r, s, c, rd, res, aux);
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

// Add the kernels of one tiled row pass (segments, then tiles) to a launch sink.
template <class Op, class Sink>
int tile_pass(const TilePlan &p, Op &op, Sink &&sink) {
    const uint32_t *ptr = p.ptr.as<uint32_t>();
    const uint32_t *idx = p.idx.as<uint32_t>();
    const uint2 *tiles = p.tiles.as<uint2>();
    const uint2 *seg_range = p.seg_range.as<uint2>();
    float2 *segs = p.segs.as<float2>();
    const float2 *csegs = segs;
    double *partials = p.partials.as<double>();
    if (p.nsegs) {
        uint32_t nsegs = p.nsegs;
        void *a_seg[] = {&idx, &seg_range, &nsegs, &op, &segs};
        OLV_TRY(sink((const void *)k_row_segments<Op>,
                     dim3((nsegs + kBlock / 32 - 1) / (kBlock / 32)), dim3(kBlock), a_seg));
    }
    uint32_t ntiles = p.ntiles, n = p.n;
    void *a_t[] = {&ptr, &idx, &tiles, &ntiles, &n, &csegs, &op, &partials};
    OLV_TRY(sink((const void *)k_row_tiles<Op>, dim3(kTileCTAs), dim3(kBlock), a_t));
    return OLV_OK;
}

}  // namespace olv
