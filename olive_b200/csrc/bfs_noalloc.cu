// olv_bfs_noalloc: BFS levels through caller-provided device buffers, with
// no device or host allocation inside the call.
//
// Some callers cannot allocate: a host that owns every byte of device memory
// through its own pool and forbids cudaMalloc in plugins, code that runs where
// an allocation would synchronise the device or fail (a memory-capped process
// at the edge of its budget), or a runtime that must not create handles on
// its own.  They pass the CSR and the level array they already own; the
// engine's scratch (two frontier queues, the hub-piece list and the control
// block) lives in one file-scope __device__ array, g_noalloc_scratch, of a
// fixed size: graphs of at most kNoAllocMaxV vertices and kNoAllocMaxE edges
// (about 8.6 MB, held on every GPU that loads the library until the process
// exits).
//
// The traversal is the engine's push (top-down) advance only: the pull
// direction needs the reverse graph, which this entry point may not build.
// Every call on a device shares the one scratch array, so calls whose work
// overlaps on the GPU (different streams, or host threads) race; serialise
// them.  The first call on each device resolves the scratch address with
// cudaGetSymbolAddress (with that device current).  Under CUDA's lazy module
// loading that first call also loads the library's device code on the device
// and so commits the fixed scratch there: a memory-capped caller should make
// its first call at initialisation time (and before any stream capture), after
// which calls commit nothing.
//
// Every caller pointer must be device (or managed) memory of the current
// device: memory of another GPU would be dereferenced by kernels that run
// here, so such a call is rejected before anything is launched.
#include <mutex>

#include "olive_b200/olv_advance.cuh"
#include "olv_internal.cuh"

namespace olv {

constexpr uint32_t kNoAllocMaxV = 1u << 20;          // 1,048,576 vertices
constexpr uint64_t kNoAllocMaxE = 1ull << 24;        // 16,777,216 edges
constexpr uint32_t kNoAllocHub = 1024;               // rows longer than this are split
constexpr uint32_t kNoAllocPiece = 1024;             // edges per piece
constexpr uint64_t kNoAllocMaxPieces = kNoAllocMaxE / kNoAllocPiece + kNoAllocMaxE / kNoAllocHub + 16;

struct NoAllocScratch {
    TravCtl ctl;
    uint32_t pad[64 - (sizeof(TravCtl) / 4) % 64];
    uint32_t q0[kNoAllocMaxV];
    uint32_t q1[kNoAllocMaxV];
    uint2 pieces[kNoAllocMaxPieces];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// kernels shared with olv_bfs (bfs.cu)
__global__ void k_fill_i32(int32_t *__restrict__ a, uint32_t n, int32_t x);
__global__ void k_bfs_init(TravCtl *c, int32_t *level, uint32_t *q0, const uint32_t *rowptr,
                           uint32_t src, unsigned long long E);
__global__ void k_bfs_begin(TravCtl *c, uint32_t V, float alpha, float beta);
__global__ void k_bfs_end(TravCtl *c, cudaGraphConditionalHandle h, int use_cond, uint32_t V);

struct NoAllocBfsOp {
    using SV = uint32_t;
    static constexpr int kMinBlocks = 1;   // CTAs per SM the advance must fit
    static constexpr bool kHasFar = false;
    static constexpr bool kPacked = false;
    const uint32_t *rowptr;
    uint32_t V;
    int32_t *level;
    int next;
    unsigned long long acc;
    unsigned long long *m_next;
    struct Pre {
        int lvl;
    };
    __device__ __forceinline__ void begin(TravCtl *c) {
        level = static_cast<int32_t *>(c->vdata);
        next = (int)c->level + 1;
        acc = 0;
        m_next = &c->m_next;
    }
    __device__ __forceinline__ uint32_t src_value(uint32_t) const { return 0; }
    __device__ __forceinline__ bool on_input(uint32_t) const { return true; }
    __device__ __forceinline__ Pre prepare(uint32_t, uint32_t, uint32_t v) const {
        return Pre{__ldcg(&level[v])};
    }
    // claims first (all issued before any result is used), then the outcomes
    template <int N>
    __device__ __forceinline__ void apply_n(const Pre (&p)[N], const uint32_t (&v)[N],
                                            int (&act)[N]) {
        int r[N];
#pragma unroll
        for (int j = 0; j < N; j++) {
            act[j] = act[j] && p[j].lvl == kInf;
            r[j] = act[j] ? atomicCAS(&level[v[j]], kInf, next) : 0;
        }
#pragma unroll
        for (int j = 0; j < N; j++) act[j] = act[j] && r[j] == kInf;
    }
    __device__ __forceinline__ void on_push(bool p, uint32_t v) {
        if (p) acc += __ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]);
    }
    __device__ __forceinline__ void flush(unsigned long long) { warp_add64(acc, m_next); }
};

// The caller's CSR is checked on the device before the traversal touches it:
// rowptr[0] == 0, rowptr[V] == E, rows non-decreasing, every column < V.
__global__ void k_noalloc_check(const uint32_t *__restrict__ rowptr,
                                const uint32_t *__restrict__ col, uint32_t V,
                                unsigned long long E, TravCtl *c) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (tid == 0 && (rowptr[0] != 0 || rowptr[V] != E)) atomicOr(&c->err, 4u);
    for (uint64_t v = tid; v < V; v += stride)
        if (rowptr[v + 1] < rowptr[v] || rowptr[v + 1] > E) atomicOr(&c->err, 4u);
    for (uint64_t e = tid; e < E; e += stride)
        if (col[e] >= V) atomicOr(&c->err, 8u);
}

// Device memory of device `dev`, or managed memory (reachable from any device).
static bool on_device(const void *p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[64];

static int noalloc_scratch(NoAllocScratch **out) {
    int dev = 0;
    OLV_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("olv_bfs_noalloc: device ordinal %d not supported", dev);
        return OLV_ERR_LIMIT;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
        g_noalloc_addr[dev] = p;
    }
    *out = static_cast<NoAllocScratch *>(g_noalloc_addr[dev]);
    return OLV_OK;
}

}  // namespace olv

using namespace olv;

extern "C" int olv_bfs_noalloc(const uint32_t *rowptr, const uint32_t *col, uint32_t V,
                               uint64_t E, uint32_t src, int32_t *level_out, void *stream,
                               olv_stats *st) {
    OLV_CHECK_ARG(rowptr && level_out && (col || E == 0), "olv_bfs_noalloc: null pointer");
    OLV_CHECK_ARG(V > 0, "olv_bfs_noalloc: V must be > 0");
    if (V > kNoAllocMaxV || E > kNoAllocMaxE) {
        set_error("olv_bfs_noalloc: graph of %u vertices and %llu edges exceeds the fixed "
                  "scratch (at most %u vertices and %llu edges); use olv_bfs",
                  V, (unsigned long long)E, kNoAllocMaxV, (unsigned long long)kNoAllocMaxE);
        return OLV_ERR_LIMIT;
    }
    OLV_CHECK_ARG(src < V, "olv_bfs_noalloc: source %u out of range (V=%u)", src, V);
    int dev = 0, sms = 148;
    OLV_CUDA(cudaGetDevice(&dev));
    OLV_CHECK_ARG(on_device(rowptr, dev) && on_device(level_out, dev) &&
                      (E == 0 || on_device(col, dev)),
                  "olv_bfs_noalloc: rowptr, col and level_out must be device memory of the "
                  "current device (%d)", dev);
    NoAllocScratch *sc = nullptr;
    OLV_TRY(noalloc_scratch(&sc));
    cudaStream_t s = (cudaStream_t)stream;
    OLV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    TravCtl *ctl = &sc->ctl;

    // control block starts at zero; the CSR is checked before any traversal
    OLV_CUDA(cudaMemsetAsync(ctl, 0, sizeof(TravCtl), s));
    k_noalloc_check<<<sms * 4, kBlock, 0, s>>>(rowptr, col, V, (unsigned long long)E, ctl);
    unsigned int err = 0;
    OLV_CUDA(cudaMemcpyAsync(&err, &ctl->err, sizeof err, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    if (err) {
        set_error("olv_bfs_noalloc: invalid CSR (%s%s)", (err & 4) ? "row offsets" : "",
                  (err & 8) ? (err & 4 ? ", column ids" : "column ids") : "");
        return OLV_ERR_ARG;
    }

    k_fill_i32<<<sms * 8, kBlock, 0, s>>>(level_out, V, kInf);
    k_bfs_init<<<1, 1, 0, s>>>(ctl, level_out, sc->q0, rowptr, src, (unsigned long long)E);
    AdvanceArgs a;
    a.rbeg = rowptr;
    a.rend = rowptr + 1;
    a.col = col;
    a.ctl = ctl;
    a.q0 = sc->q0;
    a.q1 = sc->q1;
    a.far0 = a.far1 = nullptr;
    a.pieces = sc->pieces;
    a.hub_degree = kNoAllocHub;
    a.piece = kNoAllocPiece;
    a.want_mode = 0;
    a.rbeg2 = a.rend2 = nullptr;
    a.want_mode2 = 0xffffffffu;
    NoAllocBfsOp op = {};
    op.rowptr = rowptr;
    op.V = V;
    const float never_pull = 0.0f, beta = 24.0f;
    int batch = 4;
    for (;;) {
        for (int i = 0; i < batch; i++) {
            k_bfs_begin<<<1, 1, 0, s>>>(ctl, V, never_pull, beta);
            k_advance_chunks<NoAllocBfsOp><<<sms * 4, kBlock, 0, s>>>(a, op);
            k_advance_pieces<NoAllocBfsOp><<<sms * 4, kBlock, 0, s>>>(a, op);
            k_bfs_end<<<1, 1, 0, s>>>(ctl, 0, 0, V);
        }
        OLV_CUDA(cudaGetLastError());
        unsigned int done = 0;
        OLV_CUDA(cudaMemcpyAsync(&done, &ctl->done, sizeof done, cudaMemcpyDeviceToHost, s));
        OLV_CUDA(cudaStreamSynchronize(s));
        if (done) break;
        if (batch < 16) batch *= 2;   // supersteps after the last are idle launches
    }
    TravCtl h;
    OLV_CUDA(cudaMemcpyAsync(&h, ctl, sizeof h, cudaMemcpyDeviceToHost, s));
    OLV_CUDA(cudaStreamSynchronize(s));
    if (h.err) {
        set_error("olv_bfs_noalloc: device-side check failed (code %u)", h.err);
        return OLV_ERR_STATE;
    }
    if (st) {
        st->iterations = h.steps;
        st->pull_steps = 0;
        st->vertices_reached = h.reached;
        st->edges_traversed = h.edges_traversed;
        st->edges_relaxed = h.edges_traversed;
        st->residual = 0;
        st->device_ms = 0;
    }
    return OLV_OK;
}
