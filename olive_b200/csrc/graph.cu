// Graph residency: upload / generate a CSR, build the reverse graph on the
// device, error plumbing.  Replaces Oliver::readGraph (oliver.h:190-202),
// GRD<T> (grd.h:43-170) and the CSR container of csrGraph.h:55-84.
#include <cub/cub.cuh>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "olv_graphexec.cuh"
#include "olv_internal.cuh"
#include "olv_rng.cuh"

namespace olv {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    cudaGetLastError();   // clear a non-sticky error so the handle stays usable
    return e == cudaErrorMemoryAllocation ? OLV_ERR_NOMEM : OLV_ERR_CUDA;
}

int DevBuf::ensure(size_t n) {
    if (n <= bytes && p) return OLV_OK;
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    }
    bytes = n;
    return OLV_OK;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

int resident_blocks(const olv_graph *g, const void *kernel, int *blocks) {
    int per_sm = 0;
    OLV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0));
    *blocks = (per_sm < 1 ? 1 : per_sm) * g->num_sms;
    return OLV_OK;
}

bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// ------------------------------------------------------------ kernels --
// src[e] for every CSR position e (one thread per row, rows split by warps).
__global__ void k_expand_rows(const uint32_t *__restrict__ rowptr, uint32_t V,
                              uint32_t *__restrict__ src) {
    uint32_t lane = threadIdx.x & 31;
    uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = warp; u < V; u += nwarps) {
        uint32_t b = rowptr[u], e = rowptr[u + 1];
        for (uint32_t i = b + lane; i < e; i += 32) src[i] = (uint32_t)u;
    }
}

// rowptr[v] = first position whose key >= v (keys sorted ascending).
__global__ void k_offsets_from_sorted(const uint32_t *__restrict__ keys, uint64_t n,
                                      uint32_t V, uint32_t *__restrict__ ptr) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if (keys[mid] < v) lo = mid + 1; else hi = mid;
        }
        ptr[v] = (uint32_t)lo;
    }
}

__global__ void k_offsets_from_sorted64(const unsigned long long *__restrict__ keys, uint64_t n,
                                        uint32_t V, uint32_t *__restrict__ ptr) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long key = (unsigned long long)v << 32;
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if (keys[mid] < key) lo = mid + 1; else hi = mid;
        }
        ptr[v] = (uint32_t)lo;
    }
}

template <class T>
__global__ void k_gather(const T *__restrict__ in, const uint32_t *__restrict__ idx, uint64_t n,
                         T *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[idx[i]];
}

__global__ void k_iota(uint32_t *__restrict__ a, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        a[i] = (uint32_t)i;
}

__global__ void k_low32(const unsigned long long *__restrict__ k, uint64_t n,
                        uint32_t *__restrict__ col) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        col[i] = (uint32_t)k[i];
}

// Raw RMAT draws -> permuted (src<<32|dst) keys; self-loops become ~0.
__global__ void k_rmat_keys(int scale, unsigned long long seed, unsigned long long pseed,
                            uint64_t M, unsigned long long *__restrict__ keys) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < M;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s, d;
        rmat_edge(scale, seed, i, &s, &d);
        s = permute_bits(s, scale, pseed);
        d = permute_bits(d, scale, pseed);
        keys[i] = (s == d) ? ~0ULL : (((unsigned long long)s << 32) | d);
    }
}

__global__ void k_uint_weights(uint64_t E, unsigned long long seed, uint32_t lo, uint32_t span,
                               uint32_t *__restrict__ w) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x)
        w[e] = lo + (uint32_t)((hash64(seed, e) >> 32) % span);
}

__global__ void k_degree_stats(const uint32_t *__restrict__ ptr, uint32_t V,
                               unsigned long long *__restrict__ best) {
    // best = max over v of (deg << 32 | (0xffffffff - v)): max degree, smallest id
    unsigned long long mine = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long d = ptr[v + 1] - ptr[v];
        unsigned long long key = (d << 32) | (0xffffffffULL - v);
        mine = key > mine ? key : mine;
    }
    for (int o = 16; o; o >>= 1) {
        unsigned long long t = __shfl_down_sync(0xffffffff, mine, o);
        mine = t > mine ? t : mine;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(best, mine);
}

static int grid_for(uint64_t n, int sms) {
    uint64_t b = (n + kBlock - 1) / kBlock;
    uint64_t cap = (uint64_t)sms * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Build CSC (colptr, rowidx, csc_eid, csc weights) from the resident CSR.
static int build_reverse(olv_graph *g) {
    const uint64_t E = g->E;
    const uint32_t V = g->V;
    cudaStream_t s = g->stream;
    OLV_TRY(g->colptr.ensure(((size_t)V + 1) * 4));
    OLV_TRY(g->rowidx.ensure(E * 4 + 16));
    OLV_TRY(g->csc_eid.ensure(E * 4 + 16));
    if (E == 0) {
        OLV_CUDA(cudaMemsetAsync(g->colptr.p, 0, ((size_t)V + 1) * 4, s));
        return OLV_OK;
    }
    DevBuf keys_in, keys_out, vals_in, temp;
    OLV_TRY(vals_in.ensure(E * 4));
    OLV_TRY(keys_out.ensure(E * 4));
    k_iota<<<grid_for(E, g->num_sms), kBlock, 0, s>>>(vals_in.as<uint32_t>(), E);
    size_t tb = 0;
    OLV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint32_t *)nullptr,
                                             (uint32_t *)nullptr, (const uint32_t *)nullptr,
                                             (uint32_t *)nullptr, (int64_t)E, 0, 32, s));
    OLV_TRY(temp.ensure(tb));
    // stable sort of (dst, csr position): rows of equal dst keep source order
    OLV_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb, g->col.as<uint32_t>(),
                                             keys_out.as<uint32_t>(), vals_in.as<uint32_t>(),
                                             g->csc_eid.as<uint32_t>(), (int64_t)E, 0, 32, s));
    k_offsets_from_sorted<<<grid_for((uint64_t)V + 1, g->num_sms), kBlock, 0, s>>>(
        keys_out.as<uint32_t>(), E, V, g->colptr.as<uint32_t>());
    // rowidx = source of each CSC entry
    DevBuf src;
    OLV_TRY(src.ensure(E * 4));
    k_expand_rows<<<grid_for((uint64_t)V * 32, g->num_sms), kBlock, 0, s>>>(
        g->rowptr.as<uint32_t>(), V, src.as<uint32_t>());
    k_gather<uint32_t><<<grid_for(E, g->num_sms), kBlock, 0, s>>>(
        src.as<uint32_t>(), g->csc_eid.as<uint32_t>(), E, g->rowidx.as<uint32_t>());
    if (g->weight_type != OLV_W_NONE) {
        OLV_TRY(g->csc_w.ensure(E * 4));
        k_gather<uint32_t><<<grid_for(E, g->num_sms), kBlock, 0, s>>>(
            g->w.as<uint32_t>(), g->csc_eid.as<uint32_t>(), E, g->csc_w.as<uint32_t>());
    }
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaStreamSynchronize(s));
    src.release();
    keys_out.release();
    vals_in.release();
    temp.release();
    return OLV_OK;
}

static int finish_graph(olv_graph *g) {
    OLV_TRY(build_reverse(g));
    DevBuf best;
    OLV_TRY(best.ensure(8));
    unsigned long long h[2];
    OLV_CUDA(cudaMemsetAsync(best.p, 0, 8, g->stream));
    k_degree_stats<<<grid_for(g->V, g->num_sms), kBlock, 0, g->stream>>>(
        g->rowptr.as<uint32_t>(), g->V, best.as<unsigned long long>());
    OLV_CUDA(cudaMemcpyAsync(&h[0], best.p, 8, cudaMemcpyDeviceToHost, g->stream));
    OLV_CUDA(cudaMemsetAsync(best.p, 0, 8, g->stream));
    k_degree_stats<<<grid_for(g->V, g->num_sms), kBlock, 0, g->stream>>>(
        g->colptr.as<uint32_t>(), g->V, best.as<unsigned long long>());
    OLV_CUDA(cudaMemcpyAsync(&h[1], best.p, 8, cudaMemcpyDeviceToHost, g->stream));
    OLV_CUDA(cudaStreamSynchronize(g->stream));
    g->max_out_degree = (uint32_t)(h[0] >> 32);
    g->max_in_degree = (uint32_t)(h[1] >> 32);
    OLV_CUDA(cudaMallocHost((void **)&g->host_ctl, sizeof(TravCtl)));
    OLV_CUDA(cudaEventCreate(&g->ev0));
    OLV_CUDA(cudaEventCreate(&g->ev1));
    return OLV_OK;
}

static int new_graph(olv_graph **out) {
    olv_graph *g = new (std::nothrow) olv_graph();
    if (!g) {
        set_error("host allocation failed");
        return OLV_ERR_NOMEM;
    }
    int dev = 0;
    OLV_CUDA(cudaGetDevice(&dev));
    g->device = dev;
    OLV_CUDA(cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, dev));
    OLV_CUDA(cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking));
    g->stream = g->own_stream;
    *out = g;
    return OLV_OK;
}

static int copy_in(DevBuf &dst, const void *src, size_t bytes, cudaStream_t s) {
    OLV_TRY(dst.ensure(bytes));
    if (bytes == 0) return OLV_OK;
    OLV_CUDA(cudaMemcpyAsync(dst.p, src, bytes,
                             is_device_ptr(src) ? cudaMemcpyDeviceToDevice
                                                : cudaMemcpyHostToDevice, s));
    return OLV_OK;
}

}  // namespace olv

using namespace olv;

extern "C" {

const char *olv_last_error(void) { return g_err; }
const char *olv_version(void) { return "olive_b200 0.1 (sm_100a)"; }

int olv_graph_create(const uint32_t *rowptr, const uint32_t *col, const void *weights,
                     int weight_type, uint32_t V, uint64_t E, olv_graph **out) {
    OLV_CHECK_ARG(out && rowptr, "olv_graph_create: null pointer");
    OLV_CHECK_ARG(V > 0, "olv_graph_create: V must be > 0");
    OLV_CHECK_ARG(E <= 0xffffffffULL, "olv_graph_create: E=%llu exceeds uint32 EdgeId",
                  (unsigned long long)E);
    OLV_CHECK_ARG(E == 0 || col, "olv_graph_create: null col");
    OLV_CHECK_ARG(weight_type == OLV_W_NONE || weight_type == OLV_W_U32 ||
                  weight_type == OLV_W_F32, "olv_graph_create: bad weight_type %d", weight_type);
    OLV_CHECK_ARG(weight_type == OLV_W_NONE || E == 0 || weights,
                  "olv_graph_create: null weights");
    *out = nullptr;
    olv_graph *g = nullptr;
    OLV_TRY(new_graph(&g));
    g->V = V;
    g->E = E;
    g->weight_type = weight_type;
    int r = copy_in(g->rowptr, rowptr, ((size_t)V + 1) * 4, g->stream);
    if (r == OLV_OK) r = copy_in(g->col, col, E * 4, g->stream);
    if (r == OLV_OK && weight_type != OLV_W_NONE) r = copy_in(g->w, weights, E * 4, g->stream);
    if (r == OLV_OK) {
        // validate: rowptr monotone, rowptr[V] == E, col < V
        std::vector<uint32_t> h(V + 1);
        cudaError_t e = cudaMemcpyAsync(h.data(), g->rowptr.p, ((size_t)V + 1) * 4,
                                        cudaMemcpyDeviceToHost, g->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "rowptr check", __FILE__, __LINE__);
        if (r == OLV_OK && (h[0] != 0 || h[V] != E)) {
            set_error("olv_graph_create: rowptr[0]=%u rowptr[V]=%u, expected 0 and E=%llu",
                      h[0], h[V], (unsigned long long)E);
            r = OLV_ERR_ARG;
        }
        for (uint32_t v = 0; r == OLV_OK && v < V; v++)
            if (h[v + 1] < h[v]) {
                set_error("olv_graph_create: rowptr decreases at vertex %u", v);
                r = OLV_ERR_ARG;
            }
    }
    if (r == OLV_OK && E) {
        std::vector<uint32_t> hc(E);
        cudaError_t e = cudaMemcpyAsync(hc.data(), g->col.p, E * 4, cudaMemcpyDeviceToHost,
                                        g->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "col check", __FILE__, __LINE__);
        for (uint64_t i = 0; r == OLV_OK && i < E; i++)
            if (hc[i] >= V) {
                set_error("olv_graph_create: col[%llu]=%u out of range (V=%u)",
                          (unsigned long long)i, hc[i], V);
                r = OLV_ERR_ARG;
            }
    }
    if (r == OLV_OK) r = finish_graph(g);
    if (r != OLV_OK) {
        olv_graph_destroy(g);
        return r;
    }
    *out = g;
    return OLV_OK;
}

int olv_graph_create_rmat(int scale, int edge_factor, uint64_t seed, int weight_type,
                          uint64_t wseed, olv_graph **out) {
    OLV_CHECK_ARG(out, "olv_graph_create_rmat: null out");
    OLV_CHECK_ARG(scale >= 1 && scale <= 30, "olv_graph_create_rmat: scale %d out of [1,30]",
                  scale);
    OLV_CHECK_ARG(edge_factor >= 1, "olv_graph_create_rmat: edge_factor must be >= 1");
    OLV_CHECK_ARG(weight_type == OLV_W_NONE || weight_type == OLV_W_U32,
                  "olv_graph_create_rmat: weight_type must be NONE or U32");
    const uint64_t V = 1ULL << scale;
    const uint64_t M = (uint64_t)edge_factor * V;
    if (M > 0xffffffffULL) {
        set_error("olv_graph_create_rmat: %llu draws exceed uint32 EdgeId",
                  (unsigned long long)M);
        return OLV_ERR_LIMIT;
    }
    *out = nullptr;
    olv_graph *g = nullptr;
    OLV_TRY(new_graph(&g));
    g->V = (uint32_t)V;
    g->weight_type = weight_type;
    cudaStream_t s = g->stream;
    int r = OLV_OK;
    {
        DevBuf k0, k1, temp, nsel;
        r = k0.ensure(M * 8);
        if (r == OLV_OK) r = k1.ensure(M * 8);
        if (r == OLV_OK) {
            unsigned long long pseed = seed ^ 0x5bd1e9955bd1e995ULL;
            k_rmat_keys<<<grid_for(M, g->num_sms), kBlock, 0, s>>>(
                scale, seed, pseed, M, k0.as<unsigned long long>());
            size_t tb = 0, tb2 = 0;
            cub::DeviceRadixSort::SortKeys(nullptr, tb, (const unsigned long long *)nullptr,
                                           (unsigned long long *)nullptr, (int64_t)M, 0, 64, s);
            cub::DeviceSelect::Unique(nullptr, tb2, (const unsigned long long *)nullptr,
                                      (unsigned long long *)nullptr, (uint64_t *)nullptr,
                                      (int64_t)M, s);
            r = temp.ensure(tb > tb2 ? tb : tb2);
            if (r == OLV_OK) r = nsel.ensure(8);
            if (r == OLV_OK) {
                cudaError_t e = cub::DeviceRadixSort::SortKeys(
                    temp.p, tb, k0.as<unsigned long long>(), k1.as<unsigned long long>(),
                    (int64_t)M, 0, 64, s);
                if (e == cudaSuccess)
                    e = cub::DeviceSelect::Unique(temp.p, tb2, k1.as<unsigned long long>(),
                                                  k0.as<unsigned long long>(),
                                                  nsel.as<uint64_t>(), (int64_t)M, s);
                uint64_t n = 0;
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(&n, nsel.p, 8, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) r = cuda_fail(e, "rmat sort/unique", __FILE__, __LINE__);
                if (r == OLV_OK) {
                    // drop the self-loop sentinel (sorted last)
                    unsigned long long last = 0;
                    if (n) {
                        e = cudaMemcpy(&last, k0.as<unsigned long long>() + n - 1, 8,
                                       cudaMemcpyDeviceToHost);
                        if (e != cudaSuccess) r = cuda_fail(e, "memcpy", __FILE__, __LINE__);
                        if (last == ~0ULL) n--;
                    }
                    g->E = n;
                }
                if (r == OLV_OK) r = g->rowptr.ensure((V + 1) * 4);
                if (r == OLV_OK) r = g->col.ensure(g->E * 4 + 16);
                if (r == OLV_OK) {
                    k_offsets_from_sorted64<<<grid_for(V + 1, g->num_sms), kBlock, 0, s>>>(
                        k0.as<unsigned long long>(), g->E, (uint32_t)V,
                        g->rowptr.as<uint32_t>());
                    k_low32<<<grid_for(g->E, g->num_sms), kBlock, 0, s>>>(
                        k0.as<unsigned long long>(), g->E, g->col.as<uint32_t>());
                    if (weight_type == OLV_W_U32) {
                        r = g->w.ensure(g->E * 4 + 16);
                        if (r == OLV_OK)
                            k_uint_weights<<<grid_for(g->E, g->num_sms), kBlock, 0, s>>>(
                                g->E, wseed, 1u, 255u, g->w.as<uint32_t>());
                    }
                    e = cudaGetLastError();
                    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                    if (e != cudaSuccess && r == OLV_OK)
                        r = cuda_fail(e, "rmat csr", __FILE__, __LINE__);
                }
            }
        }
    }
    if (r == OLV_OK) r = finish_graph(g);
    if (r != OLV_OK) {
        olv_graph_destroy(g);
        return r;
    }
    *out = g;
    return OLV_OK;
}

int olv_graph_destroy(olv_graph *g) {
    if (!g) return OLV_OK;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    g->rowptr.release(); g->col.release(); g->w.release();
    g->colptr.release(); g->rowidx.release(); g->csc_w.release(); g->csc_eid.release();
    g->outdeg_f.release();
    g->ws.release();
    release_pr_state(g);
    release_ppr_state(g);
    release_ms_state(g);
    release_wpr_state(g);
    release_batch_state(g);
    for (WhileGraph **wg : {&g->bfs_graph, &g->sssp_graph}) {
        if (*wg) {
            (*wg)->destroy();
            delete *wg;
            *wg = nullptr;
        }
    }
    if (g->host_ctl) cudaFreeHost(g->host_ctl);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    if (g->own_stream) cudaStreamDestroy(g->own_stream);
    delete g;
    return OLV_OK;
}

int olv_graph_info(const olv_graph *g, uint32_t *V, uint64_t *E, int *weight_type) {
    OLV_CHECK_ARG(g, "olv_graph_info: null graph");
    if (V) *V = g->V;
    if (E) *E = g->E;
    if (weight_type) *weight_type = g->weight_type;
    return OLV_OK;
}

int olv_graph_copy_csr(const olv_graph *g, uint32_t *rowptr, uint32_t *col, void *weights) {
    OLV_CHECK_ARG(g, "olv_graph_copy_csr: null graph");
    if (rowptr)
        OLV_CUDA(cudaMemcpyAsync(rowptr, g->rowptr.p, ((size_t)g->V + 1) * 4, cudaMemcpyDefault,
                                 g->stream));
    if (col && g->E)
        OLV_CUDA(cudaMemcpyAsync(col, g->col.p, g->E * 4, cudaMemcpyDefault, g->stream));
    if (weights && g->E && g->weight_type != OLV_W_NONE)
        OLV_CUDA(cudaMemcpyAsync(weights, g->w.p, g->E * 4, cudaMemcpyDefault, g->stream));
    OLV_CUDA(cudaStreamSynchronize(g->stream));
    return OLV_OK;
}

int olv_graph_set_weights_f32(olv_graph *g, const float *w) {
    OLV_CHECK_ARG(g && (w || g->E == 0), "olv_graph_set_weights_f32: null pointer");
    OLV_TRY(copy_in(g->w, w, g->E * 4, g->stream));
    g->weight_type = OLV_W_F32;
    OLV_TRY(g->csc_w.ensure(g->E * 4 + 16));
    if (g->E)
        k_gather<uint32_t><<<grid_for(g->E, g->num_sms), kBlock, 0, g->stream>>>(
            g->w.as<uint32_t>(), g->csc_eid.as<uint32_t>(), g->E, g->csc_w.as<uint32_t>());
    OLV_CUDA(cudaGetLastError());
    return OLV_OK;
}

int olv_tune_set(olv_graph *g, const char *key, double value) {
    OLV_CHECK_ARG(g && key, "olv_tune_set: null pointer");
    Tuning &t = g->tune;
    if (!strcmp(key, "hub_degree")) {
        OLV_CHECK_ARG(value >= 32 && value <= 1e9, "olv_tune_set: hub_degree out of range");
        t.hub_degree = (uint32_t)value;
        g->ws.pieces.release();
    } else if (!strcmp(key, "piece")) {
        OLV_CHECK_ARG(value >= 32 && value <= 1e9, "olv_tune_set: piece out of range");
        t.piece = (uint32_t)value;
        g->ws.pieces.release();
    } else if (!strcmp(key, "sssp_hub_degree")) {
        OLV_CHECK_ARG(value >= 32 && value <= 1e9, "olv_tune_set: sssp_hub_degree out of range");
        t.sssp_hub_degree = (uint32_t)value;
        g->ws.pieces.release();
    } else if (!strcmp(key, "sssp_piece")) {
        OLV_CHECK_ARG(value >= 32 && value <= 1e9, "olv_tune_set: sssp_piece out of range");
        t.sssp_piece = (uint32_t)value;
        g->ws.pieces.release();
    } else if (!strcmp(key, "alpha")) {
        OLV_CHECK_ARG(value > 0, "olv_tune_set: alpha must be > 0");
        t.alpha = (float)value;
    } else if (!strcmp(key, "beta")) {
        OLV_CHECK_ARG(value > 0, "olv_tune_set: beta must be > 0");
        t.beta = (float)value;
    } else if (!strcmp(key, "sssp_delta")) {
        OLV_CHECK_ARG(value >= 0 && value < 2147483647.0, "olv_tune_set: bad sssp_delta");
        t.sssp_delta = (uint32_t)value;
    } else if (!strcmp(key, "sssp_pull")) {
        t.sssp_pull = value != 0;
    } else if (!strcmp(key, "sssp_relabel")) {
        t.sssp_relabel = value != 0;
    } else if (!strcmp(key, "sssp_sub")) {
        OLV_CHECK_ARG(value >= 0 && value < 2147483647.0, "olv_tune_set: bad sssp_sub");
        t.sssp_sub = (uint32_t)value;
    } else if (!strcmp(key, "sssp_sub_buckets")) {
        OLV_CHECK_ARG(value >= 0 && value < 2147483647.0, "olv_tune_set: bad sssp_sub_buckets");
        t.sssp_sub_buckets = (uint32_t)value;
    } else if (!strcmp(key, "sssp_spt")) {
        OLV_CHECK_ARG(value == 1 || value == 2 || value == 4 || value == 8,
                      "olv_tune_set: sssp_spt must be 1, 2, 4 or 8");
        t.sssp_spt = (uint32_t)value;
    } else if (!strcmp(key, "sssp_tail_delta")) {
        OLV_CHECK_ARG(value >= 0 && value < 2147483647.0, "olv_tune_set: bad sssp_tail_delta");
        t.sssp_tail_delta = (uint32_t)value;
    } else if (!strcmp(key, "sssp_pull_split")) {
        OLV_CHECK_ARG(value == 0 || value == 4 || value == 8 || value == 16 || value == 32,
                      "olv_tune_set: sssp_pull_split must be 0, 4, 8, 16 or 32");
        t.sssp_pull_split = (uint32_t)value;
    } else if (!strcmp(key, "sssp_pull_direct")) {
        t.sssp_pull_direct = value != 0;
    } else if (!strcmp(key, "sssp_route")) {
        t.sssp_route = value != 0;
    } else if (!strcmp(key, "sssp_fuse_end")) {
        t.sssp_fuse_end = value != 0;
    } else if (!strcmp(key, "pr_tile_u")) {
        const uint32_t u = (uint32_t)value;
        OLV_CHECK_ARG(value >= 1 && value <= 32 && (u & (u - 1)) == 0,
                      "olv_tune_set: pr_tile_u must be a power of two in [1, 32]");
        if (u != t.pr_tile_u) {   // the row plans are rebuilt on their next use
            t.pr_tile_u = u;
            release_pr_state(g);
            release_wpr_state(g);
        }
    } else if (!strcmp(key, "ms_alpha")) {
        OLV_CHECK_ARG(value > 0, "olv_tune_set: ms_alpha must be > 0");
        t.ms_alpha = (float)value;
    } else if (!strcmp(key, "use_graphs")) {
        t.use_graphs = value != 0;
    } else if (!strcmp(key, "batch_cluster")) {
        OLV_CHECK_ARG(value == 0 || value == 1 || value == 8 || value == 16,
                      "olv_tune_set: batch_cluster must be 0, 1, 8 or 16");
        t.batch_cluster = (int)value;
    } else if (!strcmp(key, "levels_per_sync")) {
        OLV_CHECK_ARG(value >= 1 && value <= 1024, "olv_tune_set: levels_per_sync out of range");
        t.levels_per_sync = (int)value;
    } else {
        set_error("olv_tune_set: unknown key '%s'", key);
        return OLV_ERR_ARG;
    }
    // launch parameters are baked into the cached superstep graphs
    for (WhileGraph *wg : {g->bfs_graph, g->sssp_graph})
        if (wg) wg->destroy();
    release_ms_state(g);
    return OLV_OK;
}

int olv_tune_get(const olv_graph *g, const char *key, double *value) {
    OLV_CHECK_ARG(g && key && value, "olv_tune_get: null pointer");
    const Tuning &t = g->tune;
    if (!strcmp(key, "hub_degree")) *value = t.hub_degree;
    else if (!strcmp(key, "piece")) *value = t.piece;
    else if (!strcmp(key, "alpha")) *value = t.alpha;
    else if (!strcmp(key, "beta")) *value = t.beta;
    else if (!strcmp(key, "sssp_delta")) *value = t.sssp_delta;
    else if (!strcmp(key, "sssp_pull")) *value = t.sssp_pull;
    else if (!strcmp(key, "sssp_relabel")) *value = t.sssp_relabel;
    else if (!strcmp(key, "sssp_sub")) *value = t.sssp_sub;
    else if (!strcmp(key, "sssp_sub_buckets")) *value = t.sssp_sub_buckets;
    else if (!strcmp(key, "sssp_spt")) *value = t.sssp_spt;
    else if (!strcmp(key, "sssp_fuse_end")) *value = t.sssp_fuse_end;
    else if (!strcmp(key, "sssp_route")) *value = t.sssp_route;
    else if (!strcmp(key, "sssp_pull_direct")) *value = t.sssp_pull_direct;
    else if (!strcmp(key, "sssp_pull_split")) *value = t.sssp_pull_split;
    else if (!strcmp(key, "sssp_tail_delta")) *value = t.sssp_tail_delta;
    else if (!strcmp(key, "sssp_hub_degree")) *value = t.sssp_hub_degree;
    else if (!strcmp(key, "sssp_piece")) *value = t.sssp_piece;
    else if (!strcmp(key, "ms_alpha")) *value = t.ms_alpha;
    else if (!strcmp(key, "pr_tile_u")) *value = t.pr_tile_u;
    else if (!strcmp(key, "use_graphs")) *value = t.use_graphs;
    else if (!strcmp(key, "batch_cluster")) *value = t.batch_cluster;
    else if (!strcmp(key, "levels_per_sync")) *value = t.levels_per_sync;
    else {
        set_error("olv_tune_get: unknown key '%s'", key);
        return OLV_ERR_ARG;
    }
    return OLV_OK;
}

int olv_set_stream(olv_graph *g, void *stream) {
    OLV_CHECK_ARG(g, "olv_set_stream: null graph");
    g->stream = stream ? (cudaStream_t)stream : g->own_stream;
    return OLV_OK;
}

int olv_graph_max_degree_vertex(const olv_graph *g, uint32_t *v, uint32_t *deg) {
    OLV_CHECK_ARG(g && v, "olv_graph_max_degree_vertex: null pointer");
    DevBuf best;
    OLV_TRY(best.ensure(8));
    unsigned long long h = 0;
    OLV_CUDA(cudaMemsetAsync(best.p, 0, 8, g->stream));
    k_degree_stats<<<grid_for(g->V, g->num_sms), kBlock, 0, g->stream>>>(
        g->rowptr.as<uint32_t>(), g->V, best.as<unsigned long long>());
    OLV_CUDA(cudaMemcpyAsync(&h, best.p, 8, cudaMemcpyDeviceToHost, g->stream));
    OLV_CUDA(cudaStreamSynchronize(g->stream));
    *v = 0xffffffffu - (uint32_t)(h & 0xffffffffULL);
    if (deg) *deg = (uint32_t)(h >> 32);
    return OLV_OK;
}

}  // extern "C"
