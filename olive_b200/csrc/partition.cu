// One rank's share of a 1-D vertex partition, for running a graph across
// GPUs (no working reference counterpart: the reference's multi-GPU engine --
// olive.h:61-199, partition.h:95-436, messageBox.h:66-105 with the random
// edge-cut of partitionStrategy.h:58-62 -- includes a missing flexible.h and
// never built).
//
// A rank owns the vertices [lo, hi) (lo a multiple of 64, so its slice of a
// bitmap is whole 64-bit words) and holds their in-edges: the rows lo..hi-1
// of the reverse graph, with global source ids.  The exchange between ranks
// happens on the host side of the caller (olive_b200/parallel.py: NCCL
// all-gathers over NVLink, gloo in the CPU tests); these steps only read
// replicated inputs and write the rank's own slice:
//   olv_part_bfs_step  a bottom-up BFS level over the owned unvisited
//                      vertices (olv::k_pull_first_rows / k_pull_first_long:
//                      a vertex stops at its first in-neighbour in the
//                      replicated frontier bitmap), writing their levels and
//                      the rank's words of the next frontier;
//   olv_part_pr_step   a PageRank iteration over the owned rows from the
//                      replicated contribution vector r/outdeg: fixed-order
//                      compensated FP32 sums (a warp per row, lanes in a
//                      fixed stride, a fixed shuffle tree), the new ranks and
//                      contributions, and FP64 sums of |r' - r| and of the
//                      dangling ranks (per-CTA partials folded in order).
#include <vector>

#include "olive_b200/olv_advance.cuh"
#include "olv_internal.cuh"

struct olv_part {
    uint32_t V = 0, lo = 0, hi = 0;
    uint64_t E = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    olv::DevBuf colptr, rowidx, outdeg, ctl, rows, scratch, partials;
};

namespace olv {

constexpr int kPartCTAs = 148 * 4;   // fixed grid of the PageRank step (fixed partial order)

// BFS level as a first-contribution pull Op (olv_advance.cuh's protocol).
struct PartBfsOp {
    static constexpr int kMinBlocks = 4;
    static constexpr bool kFirstHit = true;
    using Acc = int32_t;
    const uint64_t *frontier;   // V bits
    int32_t *level;             // owned vertices
    uint64_t *next;             // owned words of the next frontier
    uint32_t lo;
    int32_t next_level;
    __device__ __forceinline__ bool row_wanted(uint32_t r) const { return level[r] == kInf; }
    __device__ __forceinline__ bool contributes(uint32_t u, uint32_t, int32_t &x) const {
        x = next_level;
        return passes(u);
    }
    __device__ __forceinline__ bool passes(uint32_t u) const {
        return (__ldg(&frontier[u >> 6]) >> (u & 63)) & 1;
    }
    __device__ __forceinline__ int32_t contribution(uint32_t, uint32_t) const { return next_level; }
    __device__ __forceinline__ void reduce_row(uint32_t r, int32_t x) { level[r] = x; }
    __device__ __forceinline__ bool mark(uint32_t r) {
        const uint32_t b = r + (lo & 63);   // lo is a multiple of 64: bit r of the slice
        atomicOr(reinterpret_cast<unsigned long long *>(&next[b >> 6]), 1ull << (b & 63));
        return true;
    }
};

__global__ void k_part_ctl(TravCtl *c) {
    TravCtl t = {};
    t.mode = 1;   // the pull kernels' want_mode
    *c = t;
}

// PageRank rows: warp per row, lanes stride the in-edges, compensated sums.
__global__ void __launch_bounds__(kBlock)
k_part_pr(const uint32_t *__restrict__ colptr, const uint32_t *__restrict__ rowidx,
          const uint32_t *__restrict__ outdeg, uint32_t n, const float *__restrict__ contrib,
          float base, float a_hi, float a_lo, float *__restrict__ rank,
          float *__restrict__ contrib_out, double *__restrict__ partials) {
    __shared__ double s_res[kBlock / 32], s_dang[kBlock / 32];
    const uint32_t lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    double res = 0, dang = 0;
    for (uint32_t r = warp; r < n; r += nwarps) {
        const uint32_t b = __ldg(&colptr[r]), e = __ldg(&colptr[r + 1]);
        float s = 0.0f, c = 0.0f;
        for (uint32_t j = b + lane; j < e; j += 32) {
            const float x = __ldg(&contrib[__ldg(&rowidx[j])]);
            const float t = s + x;
            const float bp = t - s;
            c += (s - (t - bp)) + (x - bp);
            s = t;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {   // fixed tree: (s, c) pairs
            const float so = __shfl_down_sync(0xffffffffu, s, o);
            const float co = __shfl_down_sync(0xffffffffu, c, o);
            const float t = s + so;
            const float bp = t - s;
            c += co + ((s - (t - bp)) + (so - bp));
            s = t;
        }
        if (lane == 0) {
            const float sum = s + c;
            const float nr = fmaf(a_hi, sum, fmaf(a_lo, sum, base));
            res += fabs((double)nr - (double)rank[r]);
            rank[r] = nr;
            const uint32_t d = outdeg[r];
            if (d) {
                contrib_out[r] = __fdiv_rn(nr, (float)d);
            } else {
                contrib_out[r] = 0.0f;
                dang += (double)nr;
            }
        }
    }
    if (lane == 0) {
        s_res[wl] = res;
        s_dang[wl] = dang;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, d = 0;
        for (int w = 0; w < kBlock / 32; w++) {
            a += s_res[w];
            d += s_dang[w];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = d;
    }
}

__global__ void k_part_fold(const double *__restrict__ partials, int n, double *out) {
    if (threadIdx.x == 0) {
        double a = 0, d = 0;
        for (int i = 0; i < n; i++) {
            a += partials[2 * i];
            d += partials[2 * i + 1];
        }
        out[0] = a;
        out[1] = d;
    }
}

}  // namespace olv

using namespace olv;

extern "C" int olv_part_create(uint32_t V, uint32_t lo, uint32_t hi, const uint32_t *colptr,
                               const uint32_t *rowidx, const uint32_t *outdeg, olv_part **out) {
    OLV_CHECK_ARG(out && colptr && outdeg, "olv_part_create: null pointer");
    OLV_CHECK_ARG(lo % 64 == 0 && lo <= hi && hi <= V,
                  "olv_part_create: need lo a multiple of 64 and lo <= hi <= V");
    const uint32_t n = hi - lo;
    std::vector<uint32_t> cp((size_t)n + 1);
    const bool cp_dev = is_device_ptr(colptr);
    OLV_CUDA(cudaMemcpy(cp.data(), colptr, ((size_t)n + 1) * 4,
                        cp_dev ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
    OLV_CHECK_ARG(cp[0] == 0, "olv_part_create: colptr must start at 0");
    for (uint32_t i = 0; i < n; i++)
        OLV_CHECK_ARG(cp[i] <= cp[i + 1], "olv_part_create: colptr decreases at row %u", i);
    const uint64_t E = cp[n];
    OLV_CHECK_ARG(rowidx || E == 0, "olv_part_create: null rowidx");
    olv_part *p = new olv_part();
    p->V = V;
    p->lo = lo;
    p->hi = hi;
    p->E = E;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, dev);
    int r = p->colptr.ensure(((size_t)n + 1) * 4);
    if (r == OLV_OK) r = p->rowidx.ensure(E * 4 + 16);
    if (r == OLV_OK) r = p->outdeg.ensure((size_t)n * 4 + 16);
    if (r == OLV_OK) r = p->ctl.ensure(sizeof(TravCtl));
    if (r == OLV_OK) r = p->rows.ensure((size_t)n * 4 + 16);   // the first-hit pull's long rows
    if (r == OLV_OK) r = p->scratch.ensure((size_t)n * 4 + 16);
    if (r == OLV_OK) r = p->partials.ensure((size_t)kPartCTAs * 16 + 32);
    if (r != OLV_OK) {
        delete p;
        return r;
    }
    cudaError_t e = cudaMemcpy(p->colptr.p, cp.data(), ((size_t)n + 1) * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && E)
        e = cudaMemcpy(p->rowidx.p, rowidx, E * 4, cudaMemcpyDefault);
    if (e == cudaSuccess) e = cudaMemcpy(p->outdeg.p, outdeg, (size_t)n * 4, cudaMemcpyDefault);
    if (e != cudaSuccess) {
        delete p;
        return cuda_fail(e, "olv_part_create", __FILE__, __LINE__);
    }
    // every source id must be a vertex of the graph
    std::vector<uint32_t> ri(E ? E : 1);
    if (E) OLV_CUDA(cudaMemcpy(ri.data(), p->rowidx.p, E * 4, cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < E; i++)
        if (ri[i] >= V) {
            delete p;
            set_error("olv_part_create: source id %u out of range (V=%u)", ri[i], V);
            return OLV_ERR_ARG;
        }
    *out = p;
    return OLV_OK;
}

extern "C" int olv_part_destroy(olv_part *p) {
    delete p;
    return OLV_OK;
}

extern "C" int olv_part_set_stream(olv_part *p, void *stream) {
    OLV_CHECK_ARG(p, "olv_part_set_stream: null pointer");
    p->stream = (cudaStream_t)stream;
    return OLV_OK;
}

extern "C" int olv_part_bfs_step(olv_part *p, const uint64_t *frontier, int32_t *level,
                                 int32_t next_level, uint64_t *next, uint64_t *found) {
    OLV_CHECK_ARG(p && frontier && level && next, "olv_part_bfs_step: null pointer");
    OLV_CHECK_ARG(is_device_ptr(frontier) && is_device_ptr(level) && is_device_ptr(next),
                  "olv_part_bfs_step: frontier, level and next must be device memory");
    cudaStream_t s = p->stream;
    const uint32_t n = p->hi - p->lo;
    const size_t words = ((size_t)n + 63) / 64;
    OLV_CUDA(cudaMemsetAsync(next, 0, words * 8, s));
    TravCtl *ctl = p->ctl.as<TravCtl>();
    k_part_ctl<<<1, 1, 0, s>>>(ctl);
    PullArgs a;
    a.colptr = p->colptr.as<uint32_t>();
    a.rowidx = p->rowidx.as<uint32_t>();
    a.ctl = ctl;
    a.want_mode = 1;
    a.n = n;
    a.pieces = reinterpret_cast<uint2 *>(p->rows.p);   // long-row list (uint32 entries)
    a.qout = p->scratch.as<uint32_t>();                // newly visited (counted)
    PartBfsOp op{frontier, level, next, p->lo, next_level};
    const unsigned grid = (unsigned)p->num_sms * 4;
    k_pull_first_rows<PartBfsOp><<<grid, kBlock, 0, s>>>(a, op);
    k_pull_first_long<PartBfsOp><<<grid, kBlock, 0, s>>>(a, op);
    OLV_CUDA(cudaGetLastError());
    TravCtl h;
    OLV_CUDA(cudaMemcpyAsync(&h, ctl, sizeof h, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    if (found) *found = h.qsize[1];
    return OLV_OK;
}

extern "C" int olv_part_pr_step(olv_part *p, const float *contrib, double base, double alpha,
                                float *rank, float *contrib_out, double *sums) {
    OLV_CHECK_ARG(p && contrib && rank && contrib_out && sums, "olv_part_pr_step: null pointer");
    OLV_CHECK_ARG(is_device_ptr(contrib) && is_device_ptr(rank) && is_device_ptr(contrib_out),
                  "olv_part_pr_step: contrib, rank and contrib_out must be device memory");
    cudaStream_t s = p->stream;
    const uint32_t n = p->hi - p->lo;
    const float a_hi = (float)alpha, a_lo = (float)(alpha - (double)a_hi);
    double *part = p->partials.as<double>();
    k_part_pr<<<kPartCTAs, kBlock, 0, s>>>(p->colptr.as<uint32_t>(), p->rowidx.as<uint32_t>(),
                                           p->outdeg.as<uint32_t>(), n, contrib, (float)base,
                                           a_hi, a_lo, rank, contrib_out, part);
    k_part_fold<<<1, 32, 0, s>>>(part, kPartCTAs, part + 2 * kPartCTAs);
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaMemcpyAsync(sums, part + 2 * kPartCTAs, 16, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    return OLV_OK;
}
