// Internal declarations shared by the translation units of libolive_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "olive_b200.h"
#include "olive_b200/olv_travctl.cuh"

namespace olv {

// ---------------------------------------------------------------- errors --
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define OLV_CUDA(call)                                                          \
    do {                                                                        \
        cudaError_t _e = (call);                                                \
        if (_e != cudaSuccess) return ::olv::cuda_fail(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define OLV_CHECK_ARG(cond, ...)                                                \
    do {                                                                        \
        if (!(cond)) { ::olv::set_error(__VA_ARGS__); return OLV_ERR_ARG; }     \
    } while (0)

#define OLV_TRY(call)                                                           \
    do { int _r = (call); if (_r != OLV_OK) return _r; } while (0)

// -------------------------------------------------------- device buffer --
// A plain owned device allocation (no host mirror: the reference's GRD<T>,
// grd.h:43-170, kept a host copy and synchronised it every superstep).
// Freed when it goes out of scope; not copyable (a copy would free twice).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    ~DevBuf() { release(); }
    int ensure(size_t n);     // grow to at least n bytes (contents not kept)
    void release();
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Where a caller's pointer lives.
bool is_device_ptr(const void *p);

// Tunables (olv_autotune writes them; defaults are set at graph creation).
struct Tuning {
    uint32_t hub_degree = 1024;   // rows longer than this are split into pieces
    uint32_t piece = 1024;        // edges per piece
    float alpha = 14.0f;          // push -> pull when m_f > m_unvisited / alpha
    float beta = 24.0f;           // pull -> push when n_f < V / beta
    uint32_t sssp_delta = 0;      // 0 = default bucket width (64)
    int sssp_pull = 1;            // SSSP: a bucket's heavy edges may go by an in-edge pull
    uint32_t sssp_hub_degree = 256;   // SSSP: rows with more edges are split into pieces
    uint32_t sssp_piece = 256;        // SSSP: edges per piece
    int sssp_relabel = 1;             // SSSP: run on vertices renumbered by in-degree
    uint32_t sssp_sub = 0;            // SSSP: light-phase sub-bucket width (0: none)
    uint32_t sssp_sub_buckets = 1;    // SSSP: heavy buckets whose light phase uses it
    uint32_t sssp_spt = 1;            // SSSP: queued sources per thread in a relax chunk
    uint32_t sssp_pull_split = 16;    // SSSP pull: renumbered rows with at most this many
                                      // in-edges a thread per vertex (0: none; 4, 8, 16, 32)
    int sssp_fuse_end = 0;            // SSSP: superstep end step in the pieces kernel's last CTA
    int sssp_route = 1;               // SSSP: the pull opens the first wide bucket (no split)
    int sssp_pull_direct = 1;         // SSSP: a first bucket with V/16 relax inputs pulls
                                      // without the collect pass
    uint32_t sssp_tail_delta = 1024;  // SSSP: width of the buckets after the first, which
                                      // relax every edge (<= delta: delta, light/heavy)
    float ms_alpha = 20.0f;       // msBFS: pull when active out-edges * ms_alpha > E
    uint32_t pr_tile_u = 8;       // PageRank / weighted PR: entries per lane the row
                                  // grouping aims at (lanes per row by row length)
    int levels_per_sync = 4;      // host loop: supersteps enqueued per check
    int use_graphs = 1;           // run supersteps inside a CUDA graph
    int batch_cluster = 1;        // batch PPR items run by thread-block clusters
};

struct Workspace {
    DevBuf level, q0, q1, pieces, ctl, mark, far0, far1, tmp, partials, fbits;
    DevBuf order, cand, cand2;      // BFS pull: in-degree-sorted vertices, candidate lists
    DevBuf pull_first;              // BFS pull: each vertex's first in-edge in pull order
    DevBuf pull_idx;                // BFS pull: in-edges sorted by source out-degree (desc)
    // SSSP: rows split light (w <= delta) | heavy, as (column, weight) pairs;
    // rowmid[u] the split point; per vertex its light and heavy ranges as
    // uint2 (one load each); the in-edges as (source, weight) pairs
    DevBuf sssp_cw, rowmid, sssp_lr, sssp_hr, sssp_crw;
    DevBuf blist;                   // SSSP: inputs of the current bucket's relax supersteps
    DevBuf hdin;                    // SSSP: per vertex (heavy out-degree, in-degree)
    // SSSP: vertices renumbered by in-degree (descending): new -> old and
    // old -> new ids, the CSR and CSC in the new ids with their weights, and
    // the distances in the new ids
    DevBuf sr_perm, sr_newid, sr_rowptr, sr_col, sr_w, sr_colptr, sr_rowidx, sr_cw, sr_dist;
    int sr_built = 0;
    uint32_t sr_vnz = 0;            // SSSP renumbered: vertices with in-degree > 0 (a prefix)
    uint32_t sr_vlong[4] = {0, 0, 0, 0};   // SSSP renumbered: vertices with in-degree > 4, 8,
                                           // 16, 32 (prefixes)
    int sssp_part_relabel = -1;     // SSSP: the partition above was built relabelled (1) or not
    uint32_t sssp_delta_built = 0;
    uint32_t n_heavy = 0, n_light = 0;
    void release() {
        level.release(); q0.release(); q1.release(); pieces.release(); ctl.release();
        fbits.release(); order.release(); cand.release(); cand2.release(); pull_idx.release();
        pull_first.release();
        sssp_cw.release(); rowmid.release(); sssp_lr.release(); sssp_hr.release();
        sssp_crw.release(); blist.release(); hdin.release();
        sssp_delta_built = 0;
        sr_perm.release(); sr_newid.release(); sr_rowptr.release(); sr_col.release();
        sr_w.release(); sr_colptr.release(); sr_rowidx.release(); sr_cw.release();
        sr_dist.release();
        sr_built = 0;
        sssp_part_relabel = -1;
        mark.release(); far0.release(); far1.release(); tmp.release(); partials.release();
    }
};

}  // namespace olv

namespace olv { struct WhileGraph; }

struct olv_graph {
    int device = 0;
    int num_sms = 148;
    uint32_t V = 0;
    uint64_t E = 0;
    int weight_type = OLV_W_NONE;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // CSR (out-edges) and CSC (in-edges), device resident
    olv::DevBuf rowptr, col, w, colptr, rowidx, csc_w, csc_eid;
    // per-vertex derived data
    olv::DevBuf outdeg_f;        // FP32 out-degree (PageRank)
    olv::Workspace ws;
    olv::Tuning tune;
    olv::TravCtl *host_ctl = nullptr;   // pinned mirror of the control block
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t max_out_degree = 0;
    uint32_t max_in_degree = 0;
    int persist_blocks = 0;              // resident CTAs of kBlock threads (all SMs)
    olv::WhileGraph *bfs_graph = nullptr;
    olv::WhileGraph *sssp_graph = nullptr;
    void *pr_state = nullptr;            // PageRank plan + graph (pagerank.cu)
    void *ppr_state = nullptr;           // K-vector personalised PageRank (ppr.cu)
    void *ms_state = nullptr;            // multi-source BFS masks + graph (msbfs.cu)
    void *wpr_state = nullptr;           // weighted PageRank row plans (wpr.cu)
    void *batch_state = nullptr;         // batch buffers kept between calls (batch.cu)
};

namespace olv {
// Resident CTAs of kBlock threads for `kernel` on all SMs (a persistent grid).
int resident_blocks(const olv_graph *g, const void *kernel, int *blocks);
void release_pr_state(olv_graph *g);
void release_ppr_state(olv_graph *g);
void release_ms_state(olv_graph *g);
void release_wpr_state(olv_graph *g);
void release_batch_state(olv_graph *g);
}
