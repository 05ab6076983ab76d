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
 * header unmodified.  The edge passes run on the engine's shared push and
 * pull templates (include/olive_b200/olv_advance.cuh; see oliverKernel.h).
 * Differences, on purpose:
 *   - GroupSize and UseScan default to 0 and true and are accepted but not
 *     needed: the expansion is load-balanced whatever the degree (SSSP.cu:148-149
 *     omits them, which did not compile against the reference);
 *   - cond receives the accumulator, not the vertex id (oliverKernel.h:112,135);
 *   - edge passes choose push or pull on the device: pull (over the reverse
 *     graph, built once in readGraph) when the source subset's out-edges reach
 *     E / pull_div, push otherwise.  A full pull reads every in-edge and
 *     costs about what a push over all edges costs, so by default (pull_div
 *     1) it runs only when the sources carry all E out-edges (edgeMap over
 *     every vertex, as PageRank.cu does: no atomics, one store per vertex);
 *     functors with the pullFirstHit opt-in pull from E / 16 (their rows stop
 *     at a contribution: first the in-neighbour with the most out-edges,
 *     which readGraph finds for every vertex, 8 bytes a vertex; then the
 *     others in CSC order).  OLIVE_DIRECTION=push|pull|auto and
 *     OLIVE_PULL_DIV override.  The result is the same either way (the
 *     reduce of every in-edge from a member), up to the order in which a
 *     non-associative reduce sees its inputs -- as in the reference, whose
 *     atomics fixed no order either;
 *   - accumulators are reset on the device, only the ones the previous pass
 *     wrote (the reference filled V values on the host and copied them every
 *     superstep, oliver.h:66,127 + grd.h:90-97);
 *   - primitives are stream-ordered on the default stream with no
 *     cudaThreadSynchronize after each; VertexSubset::size() and the print /
 *     reduce calls synchronise, as the reference's host reads did;
 *   - every kernel is grid-stride (no vertex is skipped at V > 2^24);
 *   - empty edge types (Dump_Edge) allocate nothing.
 */
#ifndef OLIVER_H
#define OLIVER_H

#include <cub/cub.cuh>
#include <stdlib.h>
#include <string.h>
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
        resetAccumulators();
        dst.clear();
        edgePass(src, dst.bits, dst.queue, dst.meta, f);
        dst.listKnown = true;
    }

    template <typename F, bool UseScan = true>
    void vertexFilter(VertexSubset &dst, const VertexSubset &src, F f) {
        assert(!src.isDense);
        assert(dst.isDense);
        dst.clear();
        olive_detail::k_vertex_filter<VertexValue, AccumValue, F>
            <<<gridV(), olive_detail::kT>>>(src.bits, src.queue, src.meta, vertexCount_,
                                            outdeg_, vertexValues_, accumulators_, dst.queue,
                                            dst.bits, dst.meta, f);
        CUDA_CHECK(cudaGetLastError());
    }

    template <typename F>
    void edgeMap(const VertexSubset &src, F f) {
        assert(!src.isDense);
        resetAccumulators();
        // the written accumulators are flagged in the engine's own bitmap and
        // listed directly into the reset list
        CUDA_CHECK(cudaMemsetAsync(mapBits_, 0, (words() ? words() : 1) * sizeof(Word)));
        const VertexSubset *s = &src;
        if (!src.listKnown) {   // e.g. the universal subset: list its members once
            olive_detail::k_meta_zero_for_list<<<1, 1>>>(srcList_.meta);
            olive_detail::k_bits_to_list<<<gridV(), 256>>>(src.bits, vertexCount_, outdeg_,
                                                           srcList_.queue, srcList_.meta);
            olive_detail::k_meta_list_done<<<1, 1>>>(srcList_.meta);
            CUDA_CHECK(cudaGetLastError());
            srcList_.bits = src.bits;   // membership for the pull
            s = &srcList_;
        }
        edgePass(*s, mapBits_, accList_, nullptr, f);
    }

    template <typename F>
    void vertexMap(const VertexSubset &src, F f) {
        olive_detail::k_vertex_map<VertexValue, AccumValue, F><<<gridV(), 256>>>(
            src.bits, src.queue, src.meta, src.isDense, vertexCount_, vertexValues_,
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

    explicit Oliver(AccumValue a) : defaultAccum_(a) { readPolicy(); }
    Oliver() : defaultAccum_(0) { readPolicy(); }

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
        CUDA_CHECK(cudaMalloc((void **)&outdeg_, (V ? V : 1) * sizeof(VertexId)));
        if (V) olive_detail::k_out_degrees<<<gridV(), 256>>>(rowptr_, vertexCount_, outdeg_);
        CUDA_CHECK(cudaMalloc((void **)&vertexValues_, (V ? V : 1) * sizeof(VertexValue)));
        CUDA_CHECK(cudaMemset(vertexValues_, 0, (V ? V : 1) * sizeof(VertexValue)));
        CUDA_CHECK(cudaMalloc((void **)&accumulators_, (V ? V : 1) * sizeof(AccumValue)));
        olive_detail::device_fill(accumulators_, V, defaultAccum_);
        if (!std::is_empty<EdgeValue>::value) {
            CUDA_CHECK(cudaMalloc((void **)&edgeValues_, (E ? E : 1) * sizeof(EdgeValue)));
            CUDA_CHECK(cudaMemset(edgeValues_, 0, (E ? E : 1) * sizeof(EdgeValue)));
        }
        // hub pieces of either direction, or the first-hit pull's list of rows
        // whose probe failed (uint32 entries, rows with two or more in-edges:
        // at most min(V, E / 2))
        const size_t np = E / olive_detail::kPiece + E / olive_detail::kHub + 16;
        const size_t npp = E / olive_detail::kPullPiece + E / olive_detail::kPullHub + 16;
        const size_t nlong = ((V < E / 2 ? V : E / 2) + 16) / 2 + 1;
        size_t npieces = np > npp ? np : npp;
        if (nlong > npieces) npieces = nlong;
        CUDA_CHECK(cudaMalloc((void **)&pieces_, npieces * sizeof(uint2)));
        CUDA_CHECK(cudaMalloc((void **)&ctl_, sizeof(olv::TravCtl)));
        CUDA_CHECK(cudaMemset(ctl_, 0, sizeof(olv::TravCtl)));
        CUDA_CHECK(cudaMalloc((void **)&mapBits_, (words() ? words() : 1) * sizeof(Word)));
        CUDA_CHECK(cudaMemset(mapBits_, 0, (words() ? words() : 1) * sizeof(Word)));
        CUDA_CHECK(cudaMalloc((void **)&accList_, (V ? V : 1) * sizeof(VertexId)));
        CUDA_CHECK(cudaMalloc((void **)&accMeta_, sizeof(olive_detail::SubsetMeta)));
        olive_detail::k_meta_set<<<1, 1>>>(accMeta_, 0, 1);   // nothing written yet
        srcList_ = VertexSubset(vertexCount_);
        ownedSrcBits_ = srcList_.bits;
        int dev = 0;
        CUDA_CHECK(cudaGetDevice(&dev));
        CUDA_CHECK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
        if (policy_ != 0 && E) buildReverse();
        CUDA_CHECK(cudaGetLastError());
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

    /** Edge-pass direction: 0 push, 1 pull, 2 by frontier size (default). */
    void setDirection(int policy, double pull_div = 1.0) {
        policy_ = policy;
        pullDiv_ = pull_div > 0 ? pull_div : 1.0;
        if (policy_ != 0 && edgeCount_ && !colptr_) buildReverse();
    }

    ~Oliver() {
        release();
        srcList_.bits = ownedSrcBits_;
        srcList_.del();
    }

private:
    VertexId vertexCount_ = 0;
    EdgeId edgeCount_ = 0;
    EdgeId *rowptr_ = nullptr;
    VertexId *col_ = nullptr;
    VertexId *outdeg_ = nullptr;
    EdgeId *colptr_ = nullptr;     // reverse graph: in-edges of v in [colptr[v], colptr[v+1])
    VertexId *rowidx_ = nullptr;   // their sources
    EdgeId *eid_ = nullptr;        // their CSR positions (edge values)
    VertexId *first_ = nullptr;    // first-hit pulls: each row's likeliest parent
    EdgeId *firstpos_ = nullptr;   // and the CSC position of that in-edge
    VertexValue *vertexValues_ = nullptr;
    AccumValue *accumulators_ = nullptr;
    EdgeValue *edgeValues_ = nullptr;
    uint2 *pieces_ = nullptr;
    olv::TravCtl *ctl_ = nullptr;
    Word *mapBits_ = nullptr;      // edgeMap: accumulators written this pass
    VertexId *accList_ = nullptr;  // accumulators written by the last pass
    olive_detail::SubsetMeta *accMeta_ = nullptr;
    VertexSubset srcList_;         // edgeMap over a flag subset without a list
    Word *ownedSrcBits_ = nullptr;
    AccumValue defaultAccum_;
    int sms_ = 148;
    int policy_ = 2;
    double pullDiv_ = 1.0;
    std::vector<VertexValue> hostValues_;

    size_t words() const { return ((size_t)vertexCount_ + 63) / 64; }
    unsigned gridV() const {
        size_t b = ((size_t)vertexCount_ + 255) / 256;
        size_t cap = (size_t)sms_ * 16;
        return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
    }

    void readPolicy() {
        const char *d = getenv("OLIVE_DIRECTION");
        if (d && !strcmp(d, "push")) policy_ = 0;
        if (d && !strcmp(d, "pull")) policy_ = 1;
        const char *q = getenv("OLIVE_PULL_DIV");
        if (q && atof(q) > 0) pullDiv_ = atof(q);
    }

    void resetAccumulators() {
        olive_detail::k_acc_reset<AccumValue><<<gridV(), 256>>>(
            accumulators_, vertexCount_, defaultAccum_, accList_, accMeta_);
        CUDA_CHECK(cudaGetLastError());
    }

    template <class Kernel>
    unsigned persistentGrid(Kernel k) {
        int per_sm = 0;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, olive_detail::kT, 0));
        return (unsigned)(sms_ * (per_sm > 0 ? per_sm : 1));
    }

    // One edge pass from the members of src (a listed subset): reduce into the
    // accumulators, flag the written vertices in dbits and list them in dlist.
    template <typename F>
    void edgePass(const VertexSubset &src, Word *dbits, VertexId *dlist,
                  olive_detail::SubsetMeta *dmeta, F f) {
        using namespace olive_detail;
        using PushT = PushOp<VertexValue, AccumValue, EdgeValue, F, true>;
        using PullT = PullOp<VertexValue, AccumValue, EdgeValue, F>;
        const int policy = colptr_ ? policy_ : 0;
        // a first-contribution pull reads far fewer in-edges than a full one,
        // so it pays off for smaller frontiers
        const double div = pull_first_hit<F>::value ? pullDiv_ * kFirstHitPullFactor : pullDiv_;
        const unsigned long long pull_edges = (unsigned long long)((double)edgeCount_ / div);
        k_edge_setup<<<1, 1>>>(ctl_, src.meta, policy, pull_edges);
        olv::AdvanceArgs a;
        a.rbeg = rowptr_;
        a.rend = rowptr_ + 1;
        a.col = col_;
        a.ctl = ctl_;
        a.q0 = src.queue;
        a.q1 = dlist;
        a.pieces = pieces_;
        a.hub_degree = kHub;
        a.piece = kPiece;
        a.want_mode = kModePush;
        PushT po{f, outdeg_, vertexValues_, accumulators_, edgeValues_, dbits};
        static unsigned push_grid = 0;
        if (!push_grid) push_grid = persistentGrid(olv::k_advance_chunks<PushT>);
        olv::k_advance_chunks<PushT><<<push_grid, kT>>>(a, po);
        olv::k_advance_pieces<PushT><<<push_grid, kT>>>(a, po);
        constexpr bool first_hit = pull_first_hit<F>::value;
        if (policy != 0) {
            olv::PullArgs p;
            p.colptr = colptr_;
            p.rowidx = rowidx_;
            p.ctl = ctl_;
            p.want_mode = kModePull;
            p.n = vertexCount_;
            p.pieces = pieces_;
            p.hub_degree = kPullHub;
            p.piece = kPullPiece;
            p.qout = dlist;
            PullT pl{f, outdeg_, eid_, src.bits, vertexValues_, accumulators_, edgeValues_, dbits};
            static unsigned pull_grid = 0;
            if constexpr (first_hit) {   // bottom-up: each row stops at its first contribution
                p.first = first_;
                p.firstpos = firstpos_;
                if (!pull_grid) pull_grid = persistentGrid(olv::k_pull_first_rows<PullT>);
                olv::k_pull_first_rows<PullT><<<pull_grid, kT>>>(p, pl);
                olv::k_pull_first_long<PullT><<<pull_grid, kT>>>(p, pl);
            } else {
                if (!pull_grid) pull_grid = persistentGrid(olv::k_pull_chunks<PullT>);
                olv::k_pull_chunks<PullT><<<pull_grid, kT>>>(p, pl);
                olv::k_pull_pieces<PullT><<<pull_grid, kT>>>(p, pl);
            }
        }
        k_edge_finish<<<gridV(), 256>>>(ctl_, dmeta, dlist, accList_, accMeta_);
        CUDA_CHECK(cudaGetLastError());
    }

    // Reverse graph (in-edges grouped by destination, each row in CSR order)
    // by a stable radix sort of (destination, CSR position) pairs.
    void buildReverse() {
        using namespace olive_detail;
        const size_t V = vertexCount_, E = edgeCount_;
        VertexId *src = nullptr, *keys = nullptr, *indeg = nullptr;
        EdgeId *pos = nullptr;
        CUDA_CHECK(cudaMalloc((void **)&colptr_, (V + 1) * sizeof(EdgeId)));
        CUDA_CHECK(cudaMalloc((void **)&rowidx_, E * sizeof(VertexId)));
        CUDA_CHECK(cudaMalloc((void **)&eid_, E * sizeof(EdgeId)));
        CUDA_CHECK(cudaMalloc((void **)&src, E * sizeof(VertexId)));
        CUDA_CHECK(cudaMalloc((void **)&keys, E * sizeof(VertexId)));
        CUDA_CHECK(cudaMalloc((void **)&pos, E * sizeof(EdgeId)));
        CUDA_CHECK(cudaMalloc((void **)&indeg, (V + 1) * sizeof(VertexId)));
        k_row_of_edge<<<gridV(), 256>>>(rowptr_, vertexCount_, src);
        k_iota<<<sms_ * 8, 256>>>(pos, E);
        int bits = 1;
        while (bits < 32 && ((size_t)1 << bits) < V) bits++;
        size_t tb = 0;
        CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb, (const VertexId *)nullptr,
                                                   (VertexId *)nullptr, (const EdgeId *)nullptr,
                                                   (EdgeId *)nullptr, (int)E, 0, bits));
        void *temp = nullptr;
        CUDA_CHECK(cudaMalloc(&temp, tb ? tb : 1));
        CUDA_CHECK(cub::DeviceRadixSort::SortPairs(temp, tb, col_, keys, pos, eid_, (int)E, 0,
                                                   bits));
        CUDA_CHECK(cudaFree(temp));
        k_gather_u32<<<sms_ * 8, 256>>>(src, eid_, E, rowidx_);
        // each row's likeliest parent, probed first by first-hit pulls
        unsigned long long *best = nullptr;
        CUDA_CHECK(cudaMalloc((void **)&best, V * sizeof(unsigned long long)));
        CUDA_CHECK(cudaMemset(best, 0, V * sizeof(unsigned long long)));
        k_first_parent_max<<<sms_ * 8, 256>>>(keys, rowidx_, outdeg_, E, best);
        CUDA_CHECK(cudaMalloc((void **)&first_, V * sizeof(VertexId)));
        CUDA_CHECK(cudaMalloc((void **)&firstpos_, V * sizeof(EdgeId)));
        k_first_parent_set<<<gridV(), 256>>>(best, rowidx_, V, first_, firstpos_);
        CUDA_CHECK(cudaFree(best));
        CUDA_CHECK(cudaMemset(indeg, 0, (V + 1) * sizeof(VertexId)));
        k_in_degrees<<<sms_ * 8, 256>>>(col_, E, indeg);
        tb = 0;
        CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, indeg, colptr_, (int)(V + 1)));
        CUDA_CHECK(cudaMalloc(&temp, tb ? tb : 1));
        CUDA_CHECK(cub::DeviceScan::ExclusiveSum(temp, tb, indeg, colptr_, (int)(V + 1)));
        CUDA_CHECK(cudaFree(temp));
        CUDA_CHECK(cudaFree(src));
        CUDA_CHECK(cudaFree(keys));
        CUDA_CHECK(cudaFree(pos));
        CUDA_CHECK(cudaFree(indeg));
        CUDA_CHECK(cudaGetLastError());
    }

    void pullVertices() {
        hostValues_.resize(vertexCount_);
        if (vertexCount_)
            CUDA_CHECK(cudaMemcpy(hostValues_.data(), vertexValues_,
                                  vertexCount_ * sizeof(VertexValue), cudaMemcpyDeviceToHost));
    }

    void release() {
        cudaFree(rowptr_);
        cudaFree(col_);
        cudaFree(outdeg_);
        cudaFree(colptr_);
        cudaFree(rowidx_);
        cudaFree(eid_);
        cudaFree(first_);
        cudaFree(firstpos_);
        cudaFree(vertexValues_);
        cudaFree(accumulators_);
        cudaFree(edgeValues_);
        cudaFree(pieces_);
        cudaFree(ctl_);
        cudaFree(mapBits_);
        cudaFree(accList_);
        cudaFree(accMeta_);
        rowptr_ = nullptr;
        col_ = nullptr;
        outdeg_ = nullptr;
        colptr_ = nullptr;
        rowidx_ = nullptr;
        eid_ = nullptr;
        first_ = nullptr;
        firstpos_ = nullptr;
        vertexValues_ = nullptr;
        accumulators_ = nullptr;
        edgeValues_ = nullptr;
        pieces_ = nullptr;
        ctl_ = nullptr;
        mapBits_ = nullptr;
        accList_ = nullptr;
        accMeta_ = nullptr;
        if (ownedSrcBits_) {
            srcList_.bits = ownedSrcBits_;
            srcList_.del();
            ownedSrcBits_ = nullptr;
        }
    }
};

#endif  // OLIVER_H
