// Graph ingest on the device: the reference's text formats parsed in parallel.
//
// Replaces the host loaders CsrGraph::fromEdgeListFile (csrGraph.h:106-171,
// fscanf per line, ~4 M edges/s) and CsrGraph::fromDimacsFile
// (csrGraph.h:177-236, fgetc per character) with:
//   1. one read of the file into pinned memory and one copy to the device;
//   2. newline positions by a device-wide selection, one thread per line;
//   3. each line parsed on the device: comment ('#', and '%' for DIMACS),
//      header "V E", or numbers;
//   4. edge list: the edge lines after the header, in file order, stably
//      sorted by source (the evident intent of the commented-out sort at
//      csrGraph.h:149; the reference attached out-of-order tuples to the wrong
//      row); the optional third column becomes a uint32 weight;
//      DIMACS: line k after the header holds vertex k-1's 1-based neighbours;
//      the stored edge count is twice the header's E (csrGraph.h:212,217);
//   5. the CSR handed to the same graph build as olv_graph_create (reverse
//      graph on the device).
// Ids outside [0, V) are counted and the file is rejected (OLV_ERR_ARG).
#include <cub/cub.cuh>
#include <stdio.h>

#include <vector>

#include "olv_internal.cuh"

namespace olv {

struct IsNewline {
    const char *buf;
    __host__ __device__ __forceinline__ bool operator()(const long long &i) const {
        return buf[i] == '\n';
    }
};

__device__ __forceinline__ bool is_blank(char ch) { return ch == ' ' || ch == '\t' || ch == '\r'; }

// Parse up to 3 unsigned decimals of the line [b, e); returns how many.
__device__ __forceinline__ int parse_line(const char *buf, long long b, long long e,
                                          unsigned long long *x, int maxn) {
    int n = 0;
    long long i = b;
    while (n < maxn) {
        while (i < e && is_blank(buf[i])) i++;
        if (i >= e || buf[i] < '0' || buf[i] > '9') break;
        unsigned long long v = 0;
        while (i < e && buf[i] >= '0' && buf[i] <= '9') v = v * 10 + (unsigned long long)(buf[i++] - '0');
        x[n++] = v;
    }
    return n;
}

// kind: 0 comment/blank, 1 data.  For data lines: first two numbers (and a
// third for edge lists), count of numbers.
__global__ void k_classify_lines(const char *__restrict__ buf, const long long *__restrict__ nl,
                                 long long nlines, int dimacs, uint8_t *__restrict__ kind,
                                 unsigned long long *__restrict__ a, unsigned long long *__restrict__ b,
                                 unsigned long long *__restrict__ c, uint32_t *__restrict__ nnum) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nlines;
         k += (long long)gridDim.x * blockDim.x) {
        const long long s = k == 0 ? 0 : nl[k - 1] + 1, e = nl[k];
        long long i = s;
        while (i < e && is_blank(buf[i])) i++;
        const bool comment = i < e && (buf[i] == '#' || (dimacs && buf[i] == '%'));
        unsigned long long x[3] = {0, 0, 0};
        int n = 0;
        if (!comment) {
            if (dimacs) {   // count every number on the line
                long long j = i;
                while (j < e) {
                    while (j < e && is_blank(buf[j])) j++;
                    if (j >= e || buf[j] < '0' || buf[j] > '9') break;
                    if (n < 3) parse_line(buf, j, e, &x[n], 1);
                    while (j < e && buf[j] >= '0' && buf[j] <= '9') j++;
                    n++;
                }
            } else {
                n = parse_line(buf, i, e, x, 3);
            }
        }
        // a DIMACS vertex line may be empty (a vertex without neighbours)
        kind[k] = comment ? 0 : (dimacs ? 1 : (n >= 2 ? 1 : 0));
        a[k] = x[0];
        b[k] = x[1];
        c[k] = n >= 3 ? x[2] : 1;
        nnum[k] = n;
    }
}

// DIMACS: write neighbours (0-based) of vertex-line k at out[off[k] ...].
__global__ void k_dimacs_fill(const char *__restrict__ buf, const long long *__restrict__ nl,
                              const long long *__restrict__ lines, uint64_t nv,
                              const uint64_t *__restrict__ off, uint32_t V,
                              uint32_t *__restrict__ col, unsigned int *__restrict__ bad) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < (long long)nv;
         k += (long long)gridDim.x * blockDim.x) {
        const long long ln = lines[k];
        const long long s = ln == 0 ? 0 : nl[ln - 1] + 1, e = nl[ln];
        uint64_t o = off[k];
        long long j = s;
        while (j < e) {
            while (j < e && is_blank(buf[j])) j++;
            if (j >= e || buf[j] < '0' || buf[j] > '9') break;
            unsigned long long v = 0;
            while (j < e && buf[j] >= '0' && buf[j] <= '9') v = v * 10 + (unsigned long long)(buf[j++] - '0');
            if (v < 1 || v > V) {
                atomicAdd(bad, 1u);
                v = 1;
            }
            col[o++] = (uint32_t)(v - 1);
        }
    }
}

__global__ void k_check_ids(const unsigned long long *__restrict__ s,
                            const unsigned long long *__restrict__ d, uint64_t n, uint64_t V,
                            unsigned int *__restrict__ bad) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        if (s[i] >= V || d[i] >= V) atomicAdd(bad, 1u);
}

__global__ void k_narrow(const unsigned long long *__restrict__ in, uint64_t n, uint32_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)in[i];
}

template <class T>
__global__ void k_gather_by(const T *__restrict__ in, const uint32_t *__restrict__ idx, uint64_t n,
                            T *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[idx[i]];
}

__global__ void k_iota32(uint32_t *__restrict__ a, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        a[i] = (uint32_t)i;
}

__global__ void k_row_offsets(const uint32_t *__restrict__ keys, uint64_t n, uint32_t V,
                              uint32_t *__restrict__ ptr) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= V;
         v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (keys[mid] < v) lo = mid + 1; else hi = mid;
        }
        ptr[v] = (uint32_t)lo;
    }
}

static int grid(uint64_t n) {
    uint64_t b = (n + kBlock - 1) / kBlock;
    return (int)(b < 1 ? 1 : (b > 8192 ? 8192 : b));
}

// Copy n device elements to the host.
template <class T>
static int d2h(T *h, const void *d, size_t n) {
    OLV_CUDA(cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost));
    return OLV_OK;
}

static int ingest(const char *path, int dimacs, olv_graph **out, uint32_t *V_out, uint64_t *E_out) {
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_error("olv_graph_load: cannot open %s", path);
        return OLV_ERR_ARG;
    }
    fseek(f, 0, SEEK_END);
    const long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *hbuf = nullptr;
    const long long B = size + 1;   // room for a final newline
    cudaError_t ce = cudaMallocHost((void **)&hbuf, (size_t)B);
    if (ce != cudaSuccess) {
        fclose(f);
        return cuda_fail(ce, "cudaMallocHost", __FILE__, __LINE__);
    }
    const size_t got = size > 0 ? fread(hbuf, 1, (size_t)size, f) : 0;
    fclose(f);
    long long n = (long long)got;
    if (n == 0 || hbuf[n - 1] != '\n') hbuf[n++] = '\n';
    DevBuf dbuf, nl, nnl, temp;
    int r = dbuf.ensure((size_t)n);
    if (r == OLV_OK) {
        ce = cudaMemcpy(dbuf.p, hbuf, (size_t)n, cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) r = cuda_fail(ce, "cudaMemcpy", __FILE__, __LINE__);
    }
    cudaFreeHost(hbuf);
    OLV_TRY(r);
    const char *buf = dbuf.as<char>();
    // newline positions
    OLV_TRY(nl.ensure((size_t)n * 8));
    OLV_TRY(nnl.ensure(8));
    cub::CountingInputIterator<long long> idx(0);
    size_t tb = 0;
    OLV_CUDA(cub::DeviceSelect::If(nullptr, tb, idx, nl.as<long long>(), nnl.as<long long>(), n,
                                   IsNewline{buf}));
    OLV_TRY(temp.ensure(tb));
    OLV_CUDA(cub::DeviceSelect::If(temp.p, tb, idx, nl.as<long long>(), nnl.as<long long>(), n,
                                   IsNewline{buf}));
    long long nlines = 0;
    OLV_TRY(d2h(&nlines, nnl.p, 1));
    DevBuf kind, A, Bv, C, nnum;
    OLV_TRY(kind.ensure((size_t)nlines + 1));
    OLV_TRY(A.ensure((size_t)nlines * 8 + 8));
    OLV_TRY(Bv.ensure((size_t)nlines * 8 + 8));
    OLV_TRY(C.ensure((size_t)nlines * 8 + 8));
    OLV_TRY(nnum.ensure((size_t)nlines * 4 + 4));
    k_classify_lines<<<grid(nlines), kBlock>>>(buf, nl.as<long long>(), nlines, dimacs,
                                               kind.as<uint8_t>(), A.as<unsigned long long>(),
                                               Bv.as<unsigned long long>(),
                                               C.as<unsigned long long>(), nnum.as<uint32_t>());
    OLV_CUDA(cudaGetLastError());
    // data lines, in file order
    DevBuf dl, ndl;
    OLV_TRY(dl.ensure((size_t)nlines * 8 + 8));
    OLV_TRY(ndl.ensure(8));
    tb = 0;
    OLV_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, idx, kind.as<uint8_t>(), dl.as<long long>(),
                                        ndl.as<long long>(), nlines));
    OLV_TRY(temp.ensure(tb));
    OLV_CUDA(cub::DeviceSelect::Flagged(temp.p, tb, idx, kind.as<uint8_t>(), dl.as<long long>(),
                                        ndl.as<long long>(), nlines));
    long long ndata = 0;
    OLV_TRY(d2h(&ndata, ndl.p, 1));
    if (ndata < 1) {
        set_error("olv_graph_load: %s has no header line", path);
        return OLV_ERR_ARG;
    }
    long long hdr = 0;
    OLV_TRY(d2h(&hdr, dl.p, 1));
    unsigned long long hV = 0, hE = 0;
    OLV_TRY(d2h(&hV, A.as<unsigned long long>() + hdr, 1));
    OLV_TRY(d2h(&hE, Bv.as<unsigned long long>() + hdr, 1));
    if (hV == 0 || hV > 0xfffffffeULL) {
        set_error("olv_graph_load: bad vertex count %llu in %s", hV, path);
        return OLV_ERR_ARG;
    }
    const uint32_t V = (uint32_t)hV;
    DevBuf rowptr, col, w;
    DevBuf bad;
    OLV_TRY(bad.ensure(8));
    OLV_CUDA(cudaMemset(bad.p, 0, 8));
    uint64_t E = 0;
    bool weighted = false;
    if (!dimacs) {
        // edge lines: data lines after the header, at most hE of them (csrGraph.h:124-146)
        long long ne = ndata - 1;
        if ((unsigned long long)ne > hE) ne = (long long)hE;
        E = (uint64_t)ne;
        if (E > 0xffffffffULL) {
            set_error("olv_graph_load: %llu edges exceed uint32 EdgeId", (unsigned long long)E);
            return OLV_ERR_LIMIT;
        }
        DevBuf s64, d64, c64, src, order, keys_out, tmp32;
        OLV_TRY(s64.ensure(E * 8 + 8));
        OLV_TRY(d64.ensure(E * 8 + 8));
        OLV_TRY(c64.ensure(E * 8 + 8));
        const long long *edge_lines = dl.as<long long>() + 1;
        // gather the three columns of the edge lines
        {
            DevBuf li;
            OLV_TRY(li.ensure(E * 4 + 4));
            k_narrow<<<grid(E), kBlock>>>((const unsigned long long *)edge_lines, E,
                                          li.as<uint32_t>());
            k_gather_by<unsigned long long><<<grid(E), kBlock>>>(
                A.as<unsigned long long>(), li.as<uint32_t>(), E, s64.as<unsigned long long>());
            k_gather_by<unsigned long long><<<grid(E), kBlock>>>(
                Bv.as<unsigned long long>(), li.as<uint32_t>(), E, d64.as<unsigned long long>());
            k_gather_by<unsigned long long><<<grid(E), kBlock>>>(
                C.as<unsigned long long>(), li.as<uint32_t>(), E, c64.as<unsigned long long>());
            // weighted when any edge line has a third column
            DevBuf n3, cnt;
            OLV_TRY(n3.ensure(E * 4 + 4));
            k_gather_by<uint32_t><<<grid(E), kBlock>>>(nnum.as<uint32_t>(), li.as<uint32_t>(), E,
                                                     n3.as<uint32_t>());
            OLV_TRY(cnt.ensure(8));
            tb = 0;
            OLV_CUDA(cub::DeviceReduce::Max(nullptr, tb, n3.as<uint32_t>(), cnt.as<uint32_t>(),
                                            (int64_t)E));
            OLV_TRY(temp.ensure(tb));
            OLV_CUDA(cub::DeviceReduce::Max(temp.p, tb, n3.as<uint32_t>(), cnt.as<uint32_t>(),
                                            (int64_t)E));
            uint32_t mx = 0;
            if (E) OLV_TRY(d2h(&mx, cnt.p, 1));
            weighted = mx >= 3;
        }
        k_check_ids<<<grid(E), kBlock>>>(s64.as<unsigned long long>(), d64.as<unsigned long long>(),
                                         E, V, bad.as<unsigned int>());
        unsigned int nbad = 0;
        OLV_TRY(d2h(&nbad, bad.p, 1));
        if (nbad) {
            set_error("olv_graph_load: %u edges with ids >= V=%u in %s", nbad, V, path);
            return OLV_ERR_ARG;
        }
        // stable sort by source: keys = src, values = file position
        OLV_TRY(src.ensure(E * 4 + 4));
        OLV_TRY(order.ensure(E * 4 + 4));
        OLV_TRY(keys_out.ensure(E * 4 + 4));
        OLV_TRY(tmp32.ensure(E * 4 + 4));
        k_narrow<<<grid(E), kBlock>>>(s64.as<unsigned long long>(), E, src.as<uint32_t>());
        k_iota32<<<grid(E), kBlock>>>(tmp32.as<uint32_t>(), E);
        tb = 0;
        OLV_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint32_t *)nullptr,
                                                 (uint32_t *)nullptr, (const uint32_t *)nullptr,
                                                 (uint32_t *)nullptr, (int64_t)E, 0, 32));
        OLV_TRY(temp.ensure(tb));
        if (E)
            OLV_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb, src.as<uint32_t>(),
                                                     keys_out.as<uint32_t>(), tmp32.as<uint32_t>(),
                                                     order.as<uint32_t>(), (int64_t)E, 0, 32));
        OLV_TRY(rowptr.ensure(((size_t)V + 1) * 4));
        OLV_TRY(col.ensure(E * 4 + 4));
        k_row_offsets<<<grid((uint64_t)V + 1), kBlock>>>(keys_out.as<uint32_t>(), E, V,
                                                         rowptr.as<uint32_t>());
        k_narrow<<<grid(E), kBlock>>>(d64.as<unsigned long long>(), E, tmp32.as<uint32_t>());
        k_gather_by<uint32_t><<<grid(E), kBlock>>>(tmp32.as<uint32_t>(), order.as<uint32_t>(), E,
                                                 col.as<uint32_t>());
        if (weighted) {
            OLV_TRY(w.ensure(E * 4 + 4));
            k_narrow<<<grid(E), kBlock>>>(c64.as<unsigned long long>(), E, tmp32.as<uint32_t>());
            k_gather_by<uint32_t><<<grid(E), kBlock>>>(tmp32.as<uint32_t>(),
                                                     order.as<uint32_t>(), E, w.as<uint32_t>());
        }
    } else {
        // vertex lines: data lines after the header; the first V of them
        long long nv = ndata - 1;
        if (nv > (long long)V) nv = V;
        DevBuf cnt64, off;
        OLV_TRY(cnt64.ensure((size_t)V * 8 + 8));
        OLV_TRY(off.ensure(((size_t)V + 1) * 8 + 8));
        OLV_CUDA(cudaMemset(cnt64.p, 0, (size_t)V * 8 + 8));
        const long long *vlines = dl.as<long long>() + 1;
        {
            DevBuf li, n32;
            OLV_TRY(li.ensure((size_t)nv * 4 + 4));
            OLV_TRY(n32.ensure((size_t)nv * 4 + 4));
            k_narrow<<<grid(nv), kBlock>>>((const unsigned long long *)vlines, (uint64_t)nv,
                                           li.as<uint32_t>());
            k_gather_by<uint32_t><<<grid(nv), kBlock>>>(nnum.as<uint32_t>(), li.as<uint32_t>(),
                                                      (uint64_t)nv, n32.as<uint32_t>());
            tb = 0;
            OLV_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, n32.as<uint32_t>(),
                                                   off.as<uint64_t>(), (int64_t)nv + 1));
            OLV_TRY(temp.ensure(tb));
            // exclusive sum over nv counts (+1 element for the total)
            OLV_CUDA(cudaMemset(n32.as<uint32_t>() + nv, 0, 4));
            OLV_CUDA(cub::DeviceScan::ExclusiveSum(temp.p, tb, n32.as<uint32_t>(),
                                                   off.as<uint64_t>(), (int64_t)nv + 1));
        }
        uint64_t total = 0;
        OLV_TRY(d2h(&total, off.as<uint64_t>() + nv, 1));
        if (total != 2 * hE) {
            set_error("olv_graph_load: DIMACS %s lists %llu neighbours, header says 2*%llu", path,
                      (unsigned long long)total, hE);
            return OLV_ERR_ARG;
        }
        E = total;
        OLV_TRY(col.ensure(E * 4 + 4));
        k_dimacs_fill<<<grid(nv), kBlock>>>(buf, nl.as<long long>(), vlines, (uint64_t)nv,
                                            off.as<uint64_t>(), V, col.as<uint32_t>(),
                                            bad.as<unsigned int>());
        unsigned int nbad = 0;
        OLV_TRY(d2h(&nbad, bad.p, 1));
        if (nbad) {
            set_error("olv_graph_load: %u neighbour ids outside [1, %u] in %s", nbad, V, path);
            return OLV_ERR_ARG;
        }
        // row offsets: off[k] for the listed vertices, total for trailing ones
        std::vector<uint64_t> hoff((size_t)nv + 1);
        OLV_TRY(d2h(hoff.data(), off.p, (size_t)nv + 1));
        std::vector<uint32_t> rp((size_t)V + 1);
        for (long long k = 0; k <= nv; k++) rp[k] = (uint32_t)hoff[k];
        for (uint64_t k = (uint64_t)nv + 1; k <= V; k++) rp[k] = (uint32_t)total;
        OLV_TRY(rowptr.ensure(((size_t)V + 1) * 4));
        OLV_CUDA(cudaMemcpy(rowptr.p, rp.data(), ((size_t)V + 1) * 4, cudaMemcpyHostToDevice));
    }
    OLV_CUDA(cudaGetLastError());
    OLV_CUDA(cudaDeviceSynchronize());
    *V_out = V;
    *E_out = E;
    return olv_graph_create(rowptr.as<uint32_t>(), col.as<uint32_t>(),
                            weighted ? w.p : nullptr, weighted ? OLV_W_U32 : OLV_W_NONE, V, E, out);
}

}  // namespace olv

using namespace olv;

// A binary CSR file of olv_graph_save: 1 = loaded, 0 = not that format.
static int load_binary_csr(const char *path, olv_graph **out, int *rc) {
    FILE *f = fopen(path, "rb");
    if (!f) return 0;
    char magic[8];
    uint64_t hdr[3];
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "OLVCSR1\n", 8) != 0) {
        fclose(f);
        return 0;
    }
    if (fread(hdr, 8, 3, f) != 3 || hdr[0] >= 0xffffffffull || hdr[1] > 0xffffffffull) {
        fclose(f);
        set_error("olv_graph_load: bad binary CSR header in %s", path);
        *rc = OLV_ERR_ARG;
        return 1;
    }
    const uint64_t V = hdr[0], E = hdr[1];
    const bool wts = hdr[2] & 1;
    std::vector<uint32_t> rp(V + 1), cl(E ? E : 1), w(wts && E ? E : 1);
    bool ok = fread(rp.data(), 4, V + 1, f) == V + 1 && fread(cl.data(), 4, E, f) == E &&
              (!wts || fread(w.data(), 4, E, f) == E);
    fclose(f);
    if (!ok) {
        set_error("olv_graph_load: truncated binary CSR file %s", path);
        *rc = OLV_ERR_ARG;
        return 1;
    }
    *rc = olv_graph_create(rp.data(), E ? cl.data() : nullptr, wts ? w.data() : nullptr,
                           wts ? OLV_W_U32 : OLV_W_NONE, (uint32_t)V, E, out);
    return 1;
}

extern "C" int olv_graph_load(const char *path, int format, olv_graph **out) {
    OLV_CHECK_ARG(path && out, "olv_graph_load: null pointer");
    OLV_CHECK_ARG(format == OLV_FMT_EDGE_LIST || format == OLV_FMT_DIMACS,
                  "olv_graph_load: bad format %d", format);
    *out = nullptr;
    int rc = OLV_OK;
    if (load_binary_csr(path, out, &rc)) return rc;
    uint32_t V = 0;
    uint64_t E = 0;
    return ingest(path, format == OLV_FMT_DIMACS, out, &V, &E);
}
