// Output writers (no reference kernel: the reference printed results with a
// host loop of fprintf calls, one per vertex, through the app's print()
// methods -- "%d\n" for BFS/SSSP levels, BFS.cu:41-43 and SSSP.cu:41-43, and
// "%f\n" for PageRank ranks, PageRank.cu:42-44).
//
// olv_write_text formats on the GPU: one pass computes every value's text
// length, a scan turns the lengths into offsets, a second pass writes the
// characters, and the host writes the buffer with one fwrite per chunk of
// 2^24 values.  "%f" is reproduced exactly as glibc's printf rounds it: the
// double x = m * 2^e is scaled by 10^6 in 128-bit integer arithmetic and
// rounded to nearest, ties to even, on the exact binary value; a negative
// value that rounds to zero keeps its sign ("-0.000000"), and infinities and
// NaNs print as "inf", "-inf", "nan", "-nan".  Finite values of magnitude
// 2^107 or more are rejected (OLV_ERR_LIMIT).
//
// olv_graph_save writes a graph as a binary CSR file ("OLVCSR1\n", uint64 V,
// E, flags, uint32 rowptr[V+1], col[E], [uint32 weights[E]]) that
// olv_graph_load and the header layer's CsrGraph::fromEdgeListFile read back.
#include <cub/cub.cuh>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "olive_b200/olv_advance.cuh"
#include "olv_internal.cuh"

namespace olv {

constexpr uint64_t kTextChunk = 1ull << 24;   // values formatted per pass

// round(|x| * 10^6) with ties to even, exactly; false when |x| >= 2^107.
__device__ __forceinline__ bool fixed6_units(double x, unsigned __int128 &q) {
    const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
    const int ex = (int)((bits >> 52) & 0x7ff);
    const unsigned long long man = bits & ((1ull << 52) - 1);
    unsigned long long m;
    int e;
    if (ex == 0) {
        m = man;
        e = -1074;
    } else {
        m = man | (1ull << 52);
        e = ex - 1075;
    }
    const unsigned __int128 P = (unsigned __int128)m * 1000000u;   // < 2^73
    if (e >= 0) {
        if (e > 54) return false;
        q = P << e;
        return true;
    }
    const int k = -e;
    if (k >= 120) {
        q = 0;
        return true;
    }
    q = P >> k;
    const unsigned __int128 rem = P & ((((unsigned __int128)1) << k) - 1);
    const unsigned __int128 half = ((unsigned __int128)1) << (k - 1);
    if (rem > half || (rem == half && (q & 1))) q += 1;
    return true;
}

__device__ __forceinline__ int u128_digits(unsigned __int128 v) {
    int n = 1;
    while (v >= 10) {
        v /= 10;
        n++;
    }
    return n;
}

__device__ __forceinline__ int u64_digits(unsigned long long v) {
    int n = 1;
    while (v >= 10) {
        v /= 10;
        n++;
    }
    return n;
}

// Text of value i (a line with its newline) into out, or only its length
// when out is null.  err gets 1 for a value outside the exact range.
__device__ int format_value(const void *vals, uint64_t i, int type, char *out, uint32_t *err) {
    if (type == OLV_TEXT_I32 || type == OLV_TEXT_U32) {
        long long v = type == OLV_TEXT_I32 ? (long long)((const int32_t *)vals)[i]
                                           : (long long)((const uint32_t *)vals)[i];
        const bool neg = v < 0;
        const unsigned long long a = neg ? (unsigned long long)(-v) : (unsigned long long)v;
        const int nd = u64_digits(a);
        const int len = (int)neg + nd + 1;
        if (out) {
            int p = 0;
            if (neg) out[p++] = '-';
            unsigned long long t = a;
            for (int d = nd - 1; d >= 0; d--) {
                out[p + d] = (char)('0' + t % 10);
                t /= 10;
            }
            out[p + nd] = '\n';
        }
        return len;
    }
    const double x = type == OLV_TEXT_F32 ? (double)((const float *)vals)[i]
                                          : ((const double *)vals)[i];
    const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
    const bool neg = bits >> 63;
    if (((bits >> 52) & 0x7ff) == 0x7ff) {   // inf / nan
        const bool nan = (bits & ((1ull << 52) - 1)) != 0;
        const char *w = nan ? "nan" : "inf";
        if (out) {
            int p = 0;
            if (neg) out[p++] = '-';
            for (int c = 0; c < 3; c++) out[p++] = w[c];
            out[p] = '\n';
        }
        return (int)neg + 4;
    }
    unsigned __int128 q;
    if (!fixed6_units(x, q)) {
        atomicOr(err, 1u);
        if (out) out[0] = '\n';
        return 1;
    }
    const unsigned __int128 ip = q / 1000000u;
    unsigned int frac = (unsigned int)(q - ip * 1000000u);
    const int nd = u128_digits(ip);
    const int len = (int)neg + nd + 1 + 6 + 1;
    if (out) {
        int p = 0;
        if (neg) out[p++] = '-';
        unsigned __int128 t = ip;
        for (int d = nd - 1; d >= 0; d--) {
            out[p + d] = (char)('0' + (int)(t % 10));
            t /= 10;
        }
        p += nd;
        out[p++] = '.';
        for (int d = 5; d >= 0; d--) {
            out[p + d] = (char)('0' + frac % 10);
            frac /= 10;
        }
        out[p + 6] = '\n';
    }
    return len;
}

__global__ void k_text_len(const void *vals, uint64_t n, int type, unsigned long long *len,
                           uint32_t *err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        len[i] = (unsigned long long)format_value(vals, i, type, nullptr, err);
}

__global__ void k_text_write(const void *vals, uint64_t n, int type,
                             const unsigned long long *off, char *buf, uint32_t *err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        format_value(vals, i, type, buf + off[i], err);
}

static size_t elem_size(int type) { return type == OLV_TEXT_F64 ? 8 : 4; }

}  // namespace olv

using namespace olv;

extern "C" int olv_write_text(const char *path, const void *values, uint64_t n, int type,
                              void *stream, uint64_t *bytes_out) {
    OLV_CHECK_ARG(path && (values || n == 0), "olv_write_text: null pointer");
    OLV_CHECK_ARG(type >= OLV_TEXT_I32 && type <= OLV_TEXT_F64, "olv_write_text: bad type %d",
                  type);
    cudaStream_t s = (cudaStream_t)stream;
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error("olv_write_text: cannot open %s", path);
        return OLV_ERR_ARG;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t es = elem_size(type);
    const bool on_dev = is_device_ptr(values);
    const uint64_t chunk = n < kTextChunk ? (n ? n : 1) : kTextChunk;
    DevBuf dvals, len, off, text, temp, err;
    char *host = nullptr;
    size_t host_cap = 0;
    uint64_t written = 0;
    int rc = OLV_OK;
    auto fail = [&](int r) {
        rc = r;
        return r;
    };
    do {
        if (!on_dev && fail(dvals.ensure(chunk * es + 16)) != OLV_OK) break;
        if (fail(len.ensure(chunk * 8 + 16)) != OLV_OK) break;
        if (fail(off.ensure(chunk * 8 + 16)) != OLV_OK) break;
        if (fail(err.ensure(16)) != OLV_OK) break;
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, (const unsigned long long *)nullptr,
                                      (unsigned long long *)nullptr, (int)chunk, s);
        if (fail(temp.ensure(tb + 16)) != OLV_OK) break;
        if (cudaMemsetAsync(err.p, 0, 4, s) != cudaSuccess) {
            rc = cuda_fail(cudaGetLastError(), "cudaMemsetAsync", __FILE__, __LINE__);
            break;
        }
        for (uint64_t b = 0; b < n && rc == OLV_OK; b += chunk) {
            const uint64_t m = n - b < chunk ? n - b : chunk;
            const void *src = (const char *)values + b * es;
            cudaError_t ce = cudaSuccess;
            if (!on_dev) {
                ce = cudaMemcpyAsync(dvals.p, src, m * es, cudaMemcpyHostToDevice, s);
                src = dvals.p;
            }
            unsigned long long *lens = len.as<unsigned long long>();
            if (ce == cudaSuccess) {
                k_text_len<<<sms * 8, kBlock, 0, s>>>(src, m, type, lens, err.as<uint32_t>());
                ce = cudaGetLastError();
            }
            if (ce == cudaSuccess)
                ce = cub::DeviceScan::ExclusiveSum(temp.p, tb, lens, off.as<unsigned long long>(),
                                                   (int)m, s);
            unsigned long long last_off = 0, last_len = 0;
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(&last_off, off.as<unsigned long long>() + (m - 1), 8,
                                     cudaMemcpyDeviceToHost, s);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(&last_len, lens + (m - 1), 8, cudaMemcpyDeviceToHost, s);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
            if (ce != cudaSuccess) {
                rc = cuda_fail(ce, "olv_write_text (lengths)", __FILE__, __LINE__);
                break;
            }
            const size_t total = (size_t)last_off + last_len;
            if (text.ensure(total + 16) != OLV_OK) {
                rc = OLV_ERR_NOMEM;
                break;
            }
            k_text_write<<<sms * 8, kBlock, 0, s>>>(src, m, type, off.as<unsigned long long>(),
                                                    text.as<char>(), err.as<uint32_t>());
            ce = cudaGetLastError();
            if (ce == cudaSuccess && total > host_cap) {
                if (host) cudaFreeHost(host);
                host = nullptr;
                ce = cudaMallocHost((void **)&host, total);
                host_cap = ce == cudaSuccess ? total : 0;
            }
            uint32_t e = 0;
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(host, text.p, total, cudaMemcpyDeviceToHost, s);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(&e, err.p, 4, cudaMemcpyDeviceToHost, s);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
            if (ce != cudaSuccess) {
                rc = cuda_fail(ce, "olv_write_text (text)", __FILE__, __LINE__);
                break;
            }
            if (e) {
                set_error("olv_write_text: a value of magnitude >= 2^107 has no exact %%f here");
                rc = OLV_ERR_LIMIT;
                break;
            }
            if (fwrite(host, 1, total, f) != total) {
                set_error("olv_write_text: write to %s failed", path);
                rc = OLV_ERR_ARG;
                break;
            }
            written += total;
        }
    } while (0);
    if (host) cudaFreeHost(host);
    if (fclose(f) != 0 && rc == OLV_OK) {
        set_error("olv_write_text: closing %s failed", path);
        rc = OLV_ERR_ARG;
    }
    if (rc == OLV_OK && bytes_out) *bytes_out = written;
    return rc;
}

extern "C" int olv_graph_save(const olv_graph *g, const char *path) {
    OLV_CHECK_ARG(g && path, "olv_graph_save: null pointer");
    const uint64_t V = g->V, E = g->E;
    const bool wts = g->weight_type == OLV_W_U32;
    std::vector<uint32_t> rp(V + 1), cl(E ? E : 1), w(wts && E ? E : 1);
    OLV_TRY(olv_graph_copy_csr(g, rp.data(), E ? cl.data() : nullptr, wts ? w.data() : nullptr));
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error("olv_graph_save: cannot open %s", path);
        return OLV_ERR_ARG;
    }
    const uint64_t hdr[3] = {V, E, wts ? 1ull : 0ull};
    bool ok = fwrite("OLVCSR1\n", 1, 8, f) == 8 && fwrite(hdr, 8, 3, f) == 3 &&
              fwrite(rp.data(), 4, V + 1, f) == V + 1 && fwrite(cl.data(), 4, E, f) == E &&
              (!wts || fwrite(w.data(), 4, E, f) == E);
    if (fclose(f) != 0) ok = false;
    if (!ok) {
        set_error("olv_graph_save: write to %s failed", path);
        return OLV_ERR_ARG;
    }
    return OLV_OK;
}
