/*
 * olive_b200 source-compatible header layer: Oliver<VertexValue, EdgeValue,
 * AccumValue>, the single-GPU engine class of the reference (oliver.h:46-249),
 * with the same methods, template parameters and functor contracts:
 *
 *   edgeFilter<F, GroupSize>(dst flags, src queue, f)   oliver.h:56-83
 *   vertexFilter<F, UseScan>(dst queue, src flags, f)   oliver.h:92-113
 *   edgeMap<F>(src flags, f)                            oliver.h:121-141
 *   vertexMap<F>(subset, f)                             oliver.h:148-170
 *   vertexReduce()                                      oliver.h:176-183
 *   readGraph(const CsrGraph<int,int>&)                 oliver.h:190-202
 *   printVertices / printEdges / getVertexCount         oliver.h:204-217
 *
 *   F::gather(VertexValue src, EdgeId outdeg, EdgeValue [&] e) -> AccumValue
 *   F::reduce(AccumValue &acc, AccumValue x)
 *   F::cond(VertexValue v, AccumValue acc) -> bool
 *   F::update(VertexValue &v, AccumValue acc)
 *   F::operator()(VertexValue &v, AccumValue acc)
 *
 * The reference apps (BFS.cu, SSSP.cu, PageRank.cu) compile against this
 * header unmodified.  Differences, on purpose:
 *   - GroupSize and UseScan default to 0 and true and are accepted but not
 *     needed: the expansion is load-balanced whatever the degree (SSSP.cu:148-149
 *     omits them, which did not compile against the reference);
 *   - cond receives the accumulator, not the vertex id (oliverKernel.h:112,135);
 *   - accumulators are reset on the device (the reference filled V values on the
 *     host and copied them every superstep, oliver.h:66,127 + grd.h:90-97);
 *   - primitives are stream-ordered on the default stream with no
 *     cudaThreadSynchronize after each; VertexSubset::size() and the print /
 *     reduce calls synchronise, as the reference's host reads did;
 *   - every kernel is grid-stride (no vertex is skipped at V > 2^24);
 *   - empty edge types (Dump_Edge) allocate nothing.
 * Kernels are in oliverKernel.h.
 */
#ifndef OLIVER_H
#define OLIVER_H

#include <type_traits>
#include <vector>

#include "commandLine.h"
#include "common.h"
#include "csrGraph.h"
#include "grd.h"
#include "logging.h"
#include "oliverKernel.h"
#include "timer.h"
#include "utils.h"
#include "vertexSubset.h"

template <typename VertexValue, typename EdgeValue, typename AccumValue>
class Oliver {
public:
    template <typename F, int GroupSize = 0>
    void edgeFilter(VertexSubset &dst, const VertexSubset &src, F f) {
        assert(!dst.isDense);
        assert(src.isDense);
        dst.clear();
        olive_detail::device_fill(accumulators_, vertexCount_, defaultAccum_);
        expand<F, true, true>(src, dst.flags, f);
    }

    template <typename F, bool UseScan = true>
    void vertexFilter(VertexSubset &dst, const VertexSubset &src, F f) {
        assert(!src.isDense);
        assert(dst.isDense);
        dst.clear();
        olive_detail::k_vertex_filter<VertexValue, AccumValue, F>
            <<<grid(), olive_detail::kT>>>(src.flags, vertexCount_, vertexValues_, accumulators_,
                                           dst.queue, dst.qSizeDevice, f);
        CUDA_CHECK(cudaGetLastError());
    }

    template <typename F>
    void edgeMap(const VertexSubset &src, F f) {
        assert(!src.isDense);
        olive_detail::device_fill(accumulators_, vertexCount_, defaultAccum_);
        expand<F, false, false>(src, nullptr, f);
    }

    template <typename F>
    void vertexMap(const VertexSubset &src, F f) {
        if (src.isDense)
            olive_detail::k_vertex_map_dense<VertexValue, AccumValue, F>
                <<<grid(), olive_detail::kT>>>(src.queue, src.qSizeDevice, vertexValues_,
                                               accumulators_, f);
        else
            olive_detail::k_vertex_map_sparse<VertexValue, AccumValue, F>
                <<<grid(), olive_detail::kT>>>(src.flags, vertexCount_, vertexValues_,
                                               accumulators_, f);
        CUDA_CHECK(cudaGetLastError());
    }

    /** Host-side reduction with VertexValue::reduce (a host method). */
    AccumValue vertexReduce() {
        pullVertices();
        AccumValue r = (AccumValue)0;
        for (VertexId i = 0; i < vertexCount_; i++) hostValues_[i].reduce(r);
        return r;
    }

    explicit Oliver(AccumValue a) : defaultAccum_(a) {}
    Oliver() : defaultAccum_(0) {}

    void readGraph(const CsrGraph<int, int> &graph) {
        release();
        vertexCount_ = graph.vertexCount;
        edgeCount_ = graph.edgeCount;
        const size_t V = vertexCount_, E = edgeCount_;
        CUDA_CHECK(cudaMalloc((void **)&rowptr_, (V + 1) * sizeof(EdgeId)));
        CUDA_CHECK(cudaMalloc((void **)&col_, (E ? E : 1) * sizeof(VertexId)));
        CUDA_CHECK(cudaMemcpy(rowptr_, graph.vertices, (V + 1) * sizeof(EdgeId),
                              cudaMemcpyHostToDevice));
        if (E)
            CUDA_CHECK(cudaMemcpy(col_, graph.edges, E * sizeof(VertexId), cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMalloc((void **)&vertexValues_, (V ? V : 1) * sizeof(VertexValue)));
        CUDA_CHECK(cudaMemset(vertexValues_, 0, (V ? V : 1) * sizeof(VertexValue)));
        CUDA_CHECK(cudaMalloc((void **)&accumulators_, (V ? V : 1) * sizeof(AccumValue)));
        if (!std::is_empty<EdgeValue>::value) {
            CUDA_CHECK(cudaMalloc((void **)&edgeValues_, (E ? E : 1) * sizeof(EdgeValue)));
            CUDA_CHECK(cudaMemset(edgeValues_, 0, (E ? E : 1) * sizeof(EdgeValue)));
        }
        const size_t np = E / olive_detail::kPiece + E / olive_detail::kHub + 16;
        CUDA_CHECK(cudaMalloc((void **)&pieces_, np * sizeof(uint2)));
        CUDA_CHECK(cudaMalloc((void **)&npieces_, sizeof(uint32_t)));
        int dev = 0, sms = 0;
        CUDA_CHECK(cudaGetDevice(&dev));
        CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        grid_ = sms * 8;
    }

    inline void printVertices() {
        pullVertices();
        for (VertexId i = 0; i < vertexCount_; i++) hostValues_[i].print();
    }

    inline void printEdges() {
        std::vector<EdgeValue> h(edgeCount_);
        if (edgeValues_ && edgeCount_)
            CUDA_CHECK(cudaMemcpy(h.data(), edgeValues_, edgeCount_ * sizeof(EdgeValue),
                                  cudaMemcpyDeviceToHost));
        for (auto &e : h) e.print();
    }

    inline VertexId getVertexCount() const { return vertexCount_; }

    /** Device arrays, for callers that run their own kernels on the state. */
    VertexValue *deviceVertexValues() const { return vertexValues_; }
    AccumValue *deviceAccumulators() const { return accumulators_; }

    ~Oliver() { release(); }

private:
    VertexId vertexCount_ = 0;
    EdgeId edgeCount_ = 0;
    EdgeId *rowptr_ = nullptr;
    VertexId *col_ = nullptr;
    VertexValue *vertexValues_ = nullptr;
    AccumValue *accumulators_ = nullptr;
    EdgeValue *edgeValues_ = nullptr;
    uint2 *pieces_ = nullptr;
    uint32_t *npieces_ = nullptr;
    AccumValue defaultAccum_;
    int grid_ = 148 * 8;
    std::vector<VertexValue> hostValues_;

    int grid() const { return grid_; }

    void pullVertices() {
        hostValues_.resize(vertexCount_);
        if (vertexCount_)
            CUDA_CHECK(cudaMemcpy(hostValues_.data(), vertexValues_,
                                  vertexCount_ * sizeof(VertexValue), cudaMemcpyDeviceToHost));
    }

    template <typename F, bool FromQueue, bool MarkDst>
    void expand(const VertexSubset &src, uint8_t *dstflags, F f) {
        olive_detail::ExpandArgs a;
        a.queue = src.queue;
        a.qsize = src.qSizeDevice;
        a.srcflags = src.flags;
        a.n = vertexCount_;
        a.rowptr = rowptr_;
        a.col = col_;
        a.dstflags = dstflags;
        a.pieces = pieces_;
        a.npieces = npieces_;
        CUDA_CHECK(cudaMemsetAsync(npieces_, 0, sizeof(uint32_t)));
        olive_detail::k_expand<VertexValue, AccumValue, EdgeValue, F, FromQueue, MarkDst>
            <<<grid(), olive_detail::kT>>>(a, vertexValues_, accumulators_, edgeValues_, f);
        olive_detail::k_expand_pieces<VertexValue, AccumValue, EdgeValue, F, MarkDst>
            <<<grid(), olive_detail::kT>>>(a, vertexValues_, accumulators_, edgeValues_, f);
        CUDA_CHECK(cudaGetLastError());
    }

    void release() {
        cudaFree(rowptr_);
        cudaFree(col_);
        cudaFree(vertexValues_);
        cudaFree(accumulators_);
        cudaFree(edgeValues_);
        cudaFree(pieces_);
        cudaFree(npieces_);
        rowptr_ = nullptr;
        col_ = nullptr;
        vertexValues_ = nullptr;
        accumulators_ = nullptr;
        edgeValues_ = nullptr;
        pieces_ = nullptr;
        npieces_ = nullptr;
    }
};

#endif  // OLIVER_H
