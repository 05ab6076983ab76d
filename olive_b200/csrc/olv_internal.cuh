// Internal declarations shared by the translation units of libolive_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "olive_b200.h"

namespace olv {

constexpr int32_t kInf = 0x7fffffff;     // unreached level / distance (BFS.cu:101, SSSP.cu:123)
constexpr int kBlock = 256;              // threads per CTA for the streaming kernels

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
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n);     // grow to at least n bytes (contents not kept)
    void release();
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Where a caller's pointer lives.
bool is_device_ptr(const void *p);

// ------------------------------------------------------------ control --
// Device-resident control block of one BFS / SSSP run.  Kernels read and
// update it, so a run needs no host round trip per superstep.
struct TravCtl {
    uint32_t qsize[2];          // entries in the two queue buffers
    uint32_t cur;               // input queue buffer of this superstep
    uint32_t level;             // BFS level of the input frontier
    uint32_t mode;              // 0 = push (top-down), 1 = pull (bottom-up)
    uint32_t done;
    uint32_t npieces;           // hub row pieces queued this superstep
    uint32_t steps;             // supersteps executed
    uint32_t pull_steps;
    uint32_t far_size[2];       // SSSP far pile buffers
    uint32_t far_cur;
    uint32_t threshold;         // SSSP near/far split distance
    uint32_t delta;
    uint32_t err;               // nonzero: a device-side check failed
    uint32_t err_info;
    uint32_t epoch;             // SSSP far-pile generation
    uint32_t far_min;           // SSSP smallest distance kept in the far pile
    uint32_t split_lo;          // SSSP: lower edge of the bucket being split
    uint32_t fb_cur;            // BFS: which frontier bitmap holds the current level
    uint32_t fb_valid;          // BFS: that bitmap is up to date
    uint32_t ncand[4];          // BFS pull: [0] candidates, [1] overflow
    uint32_t queue_stale;       // BFS: the frontier is only in the bitmap (after a pull level)
    uint32_t heavy_done;        // SSSP: heavy edges of the current bucket relaxed
    uint32_t bucket_lo;         // SSSP: lower distance edge of the current bucket
    uint32_t pull_pending;      // SSSP: the settled bucket's heavy edges go by a pull pass
    uint32_t aux_done;          // SSSP: CTAs of the collect pass that finished
    uint32_t bl_size;           // SSSP: entries in the bucket list
    uint32_t bl_over;           // SSSP: the bucket list overflowed (collect densely)
    uint32_t bucket_end;        // SSSP: upper distance edge of the current heavy bucket
    uint32_t sub_width;         // SSSP: light-phase sub-bucket width (0: none)
    uint32_t sub_buckets;       // SSSP: heavy buckets whose light phase is sub-bucketed
    uint32_t heavy_index;       // SSSP: heavy buckets started so far (0 = the first)
    unsigned long long heavy_work;  // SSSP: heavy out-edges of the collected bucket
    unsigned long long settled_in;  // SSSP: in-edges of all settled vertices
    uint32_t ms_track;          // msBFS: this push level records first-touched vertices
    uint32_t ms_touched;        // msBFS: vertices first touched by this level's push
    uint32_t ms_sparse_from;    // msBFS: first level applied sparsely (no store slot)
    uint32_t ms_cur_dense;      // msBFS: the frontier array is valid at every vertex
    unsigned long long ms_new_prev, ms_new_prev2;   // msBFS: vertices found one / two levels ago
    void *vdata;                // per-vertex result array of the run (level / dist)
    unsigned long long m_f;         // out-edges of the input frontier
    unsigned long long m_next;      // out-edges of vertices discovered this superstep
    unsigned long long m_unvisited; // out-edges of vertices not yet reached
    unsigned long long edges_traversed;
    unsigned long long edges_relaxed;
    unsigned long long reached;
    unsigned long long reached_pull;   // BFS: vertices found by this pull level
};

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
    float ms_alpha = 20.0f;       // msBFS: pull when active out-edges * ms_alpha > E
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
    void *ms_state = nullptr;            // multi-source BFS masks + graph (msbfs.cu)
    void *wpr_state = nullptr;           // weighted PageRank row plans (wpr.cu)
    void *batch_state = nullptr;         // batch buffers kept between calls (batch.cu)
};

namespace olv {
// Resident CTAs of kBlock threads for `kernel` on all SMs (a persistent grid).
int resident_blocks(const olv_graph *g, const void *kernel, int *blocks);
void release_pr_state(olv_graph *g);
void release_ms_state(olv_graph *g);
void release_wpr_state(olv_graph *g);
void release_batch_state(olv_graph *g);
}
