// Device-side control block of a frontier traversal and the engine's shared
// constants.  Used by the C ABI's kernels (olive_b200/csrc) and by the
// source-compatible header layer (include/olive), which instantiate the same
// advance templates (olv_advance.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace olv {

constexpr int32_t kInf = 0x7fffffff;     // unreached level / distance (BFS.cu:101, SSSP.cu:123)
constexpr int kBlock = 256;              // threads per CTA for the streaming kernels

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
    uint32_t end_arrive;        // CTAs of a superstep's last kernel that finished (epilogue)
    uint32_t bl_size;           // SSSP: entries in the bucket list
    uint32_t bl_over;           // SSSP: the bucket list overflowed (collect densely)
    uint32_t bucket_end;        // SSSP: upper distance edge of the current heavy bucket
    uint32_t sub_width;         // SSSP: light-phase sub-bucket width (0: none)
    uint32_t sub_buckets;       // SSSP: heavy buckets whose light phase is sub-bucketed
    uint32_t heavy_index;       // SSSP: heavy buckets started so far (0 = the first)
    uint32_t tail_width;        // SSSP: width of the buckets after the first (<= delta: delta)
    uint32_t all_edges;         // SSSP: the current bucket relaxes every edge in-bucket
    uint32_t route;             // SSSP: the pull opens the first wide bucket itself
    uint32_t direct_min;        // SSSP: a first bucket with this many relax inputs goes
                                // straight to the pull, without the collect pass (0: never)
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

}  // namespace olv
