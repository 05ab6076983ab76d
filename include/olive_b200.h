/*
 * olive_b200 -- C ABI of the B200 frontier engine (libolive_b200.so).
 *
 * The reference (ACSAlab/olive) has no FFI: its boundary is the header-only
 * C++ template class Oliver<VertexValue,EdgeValue,AccumValue> (oliver.h:46-249)
 * driven by the apps BFS.cu, SSSP.cu and PageRank.cu.  This header is the flat
 * C boundary a non-C++ caller binds (ctypes, cgo, JNI); each entry point names
 * the reference code whose result it reproduces.  The source-compatible C++
 * layer (include/olive/oliver.h) sits beside it for the reference apps.
 *
 * Conventions
 *   - Every function returns 0 (OLV_OK) or a negative OLV_ERR_* code and never
 *     aborts or throws.  olv_last_error() returns the message of the last
 *     failure on the calling thread.
 *   - Vertex ids and CSR offsets are uint32 (VertexId/EdgeId, common.h:55-59).
 *   - Pointers the caller passes may be host or device memory; the library
 *     inspects each with cudaPointerGetAttributes.  The caller owns them.  The
 *     library owns everything reachable from an olv_graph until
 *     olv_graph_destroy.
 *   - A graph handle is bound to one CUDA stream (olv_set_stream) and must be
 *     used by one host thread at a time.  Calls are stream-ordered; a call that
 *     writes a host buffer returns after the data has landed.
 */
#ifndef OLIVE_B200_H
#define OLIVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OLV_OK            0
#define OLV_ERR_ARG      -1   /* invalid argument (null pointer, id out of range, ...) */
#define OLV_ERR_CUDA     -2   /* a CUDA runtime call failed                             */
#define OLV_ERR_NOMEM    -3   /* device or host allocation failed                       */
#define OLV_ERR_TIMEOUT  -4   /* a bounded device-side wait ran out                     */
#define OLV_ERR_STATE    -5   /* call not valid in the handle's current state           */
#define OLV_ERR_LIMIT    -6   /* size beyond a documented limit                          */

/* weight_type for olv_graph_create */
#define OLV_W_NONE 0
#define OLV_W_U32  1
#define OLV_W_F32  2

/* format for olv_graph_load */
#define OLV_FMT_EDGE_LIST 0   /* "V E" then "src dst [weight]" lines, '#' comments  */
#define OLV_FMT_DIMACS    1   /* METIS / DIMACS-10 adjacency lines, 1-based ids     */

/* type for olv_write_text */
#define OLV_TEXT_I32 0   /* int32, "%d\n"                     */
#define OLV_TEXT_U32 1   /* uint32, "%u\n"                    */
#define OLV_TEXT_F32 2   /* float, "%f\n" of its double value  */
#define OLV_TEXT_F64 3   /* double, "%f\n"                    */

/* dangling_mode for olv_pagerank */
#define OLV_DANGLING_UNIFORM 0   /* redistribute dangling mass uniformly          */
#define OLV_DANGLING_LEAK    1   /* drop it, as PageRank.cu:63-75 / testPageRank */

typedef struct olv_graph olv_graph;
typedef struct olv_wpr_ctx olv_wpr_ctx;

typedef struct olv_stats {
    uint32_t iterations;        /* BFS/SSSP supersteps, PageRank iterations            */
    uint32_t pull_steps;        /* BFS levels run bottom-up                             */
    uint64_t vertices_reached;  /* BFS/SSSP: vertices with a finite result              */
    uint64_t edges_traversed;   /* sum of out-degrees of reached vertices (GTEPS basis)  */
    uint64_t edges_relaxed;     /* SSSP: out-edges pushed plus in-edges pulled          */
    double   residual;          /* PageRank: last L1 residual (FP64)                     */
    double   device_ms;         /* device time of the call (CUDA events)                */
} olv_stats;

const char *olv_last_error(void);
const char *olv_version(void);

/* ---- graph ----------------------------------------------------------------
 * Replaces Oliver::readGraph (oliver.h:190-202) + CsrGraph (csrGraph.h:55-84):
 * uploads a CSR (rowptr[V+1], col[E], optional weights[E]) to the device and
 * builds the reverse (CSC) graph on the device.  Rows need not be sorted.      */
int olv_graph_create(const uint32_t *rowptr, const uint32_t *col, const void *weights,
                     int weight_type, uint32_t V, uint64_t E, olv_graph **out);
/* Device-side RMAT generator (no reference counterpart): ef*2^scale draws with
 * (a,b,c,d) = (0.57,0.19,0.19,0.05), ids permuted by a seeded bijection,
 * self-loops and duplicates removed, CSR sorted by (src,dst).  weight_type
 * OLV_W_U32 adds weights uniform in [1,255] drawn from a stream indexed by
 * CSR position (seed wseed).                                                   */
int olv_graph_create_rmat(int scale, int edge_factor, uint64_t seed, int weight_type,
                          uint64_t wseed, olv_graph **out);
/* Load a graph file, parsed on the device (replaces CsrGraph::fromEdgeListFile,
 * csrGraph.h:106-171, and fromDimacsFile, csrGraph.h:177-236).  Edge lists are
 * stably sorted by source (the reference assumed sorted input); an optional
 * third column becomes uint32 weights.  DIMACS stores both directions (2E).
 * A file written by olv_graph_save (it starts with "OLVCSR1\n") is read as
 * that binary CSR whatever the format argument.                              */
int olv_graph_load(const char *path, int format, olv_graph **out);
int olv_graph_destroy(olv_graph *g);
int olv_graph_info(const olv_graph *g, uint32_t *V, uint64_t *E, int *weight_type);
/* Copy the CSR back (any of the pointers may be NULL). */
int olv_graph_copy_csr(const olv_graph *g, uint32_t *rowptr, uint32_t *col, void *weights);
/* Replace the FP32 edge weights (CSR order) without rebuilding the graph.   */
int olv_graph_set_weights_f32(olv_graph *g, const float *w);
/* Bind the handle to a CUDA stream (a cudaStream_t; NULL = the handle's own). */
int olv_set_stream(olv_graph *g, void *stream);
/* Maximum out-degree vertex, ties to the smallest id. */
int olv_graph_max_degree_vertex(const olv_graph *g, uint32_t *v, uint32_t *deg);
/* Engine tunables by name (no reference counterpart; the reference fixed its
 * launch shape in util::kernelConfig, utils.h:56-72, and the app's -g flag):
 *   "hub_degree"  BFS: rows longer than this are split into pieces  (1024)
 *   "piece"       BFS: edges per piece                              (1024)
 *   "sssp_hub_degree", "sssp_piece"  the same for SSSP's relax
 *                 supersteps (smaller pieces even out the CTAs' work) (256)
 *   "alpha"       BFS push->pull when m_f * alpha > m_unvisited     (14)
 *   "beta"        BFS pull->push when n_f * beta < V                (24)
 *   "sssp_delta"  SSSP width of the first bucket (and of every bucket when
 *                 sssp_tail_delta <= it), 0 = default, 24                (0)
 *   "sssp_pull"   SSSP: a settled bucket's heavy edges may be relaxed by
 *                 a pull over the in-edges of the unsettled vertices when
 *                 that reads fewer edges (1) or always by push (0)       (1)
 *   "sssp_relabel" SSSP runs on vertices renumbered by in-degree, so the
 *                 most-read distances share cache lines (1), or on the
 *                 graph's own ids (0); results are identical            (1)
 *   "sssp_sub"    SSSP: the light phase of the first heavy bucket(s) runs in
 *                 sub-buckets of this width (fewer repeated light
 *                 relaxations where that bucket holds most of the graph);
 *                 0 or >= sssp_delta: one sub-bucket per bucket          (0)
 *   "sssp_sub_buckets"  heavy buckets (from the first) that use sssp_sub (1)
 *   "sssp_spt"    queued sources per thread in a relax chunk: 1, 2, 4 or 8 (1)
 *   "sssp_pull_split"  SSSP pull: renumbered vertices with at most this
 *                 many in-edges (4, 8, 16 or 32) a thread per vertex, the
 *                 rest by edge-balanced chunks; 0: all by chunks        (16)
 *   "sssp_fuse_end"  SSSP superstep's end step run by the last CTA of the
 *                 relax pieces kernel instead of a launch of its own (0)
 *   "sssp_route"  SSSP with wide buckets after the first: the heavy pull
 *                 routes every vertex into the first of them (no split pass;
 *                 1) or leaves the far pile to a split (0)
 *   "sssp_pull_direct"  with sssp_route: a first bucket whose relax
 *                 inputs number V/16 or more goes to the pull without the
 *                 collect pass that chooses push or pull (1)
 *   "sssp_tail_delta"  width of the SSSP buckets after the first; above
 *                 sssp_delta those buckets relax every edge in-bucket and
 *                 have no heavy step (1024; 0: delta, light/heavy throughout)
 *   "ms_alpha"    msBFS pull when active out-edges * ms_alpha > E   (20)
 *   "pr_tile_u"   PageRank / weighted PageRank: entries per lane per round
 *                 the row grouping aims at (1..32, a power of two); sets
 *                 the lanes per row of the tile plans, rebuilt on change;
 *                 a weighted-PR backward needs its forward run after it (8)
 *   "use_graphs"  run supersteps inside CUDA graphs (1) or a host loop (0)
 *   "levels_per_sync" host loop: supersteps enqueued per check      (4)
 *   "batch_cluster" olv_batch_run: PPR items on thread-block clusters of
 *                 8 or 16 CTAs (1 = the largest the GPU runs), or one CTA per
 *                 item (0); the float results depend on the choice       (1) */
int olv_tune_set(olv_graph *g, const char *key, double value);
int olv_tune_get(const olv_graph *g, const char *key, double *value);
/* Autotuner: coordinate descent over hub_degree, alpha, beta (BFS), on
 * uint32-weighted graphs sssp_delta, sssp_tail_delta, sssp_hub_degree,
 * sssp_piece and sssp_sub (SSSP), pr_tile_u (PageRank, 10 iterations) and ms_alpha (msBFS from 16
 * sources), each candidate timed `reps` times (BFS / SSSP from the highest
 * out-degree vertex); the fastest values are
 * applied to the handle and, if json_path is not NULL, written to a JSON table
 * keyed by GPU name and graph shape.  olv_autotune_load applies such a table
 * when its key matches the handle (*applied = 1) and leaves the handle alone
 * otherwise.  Results stay bit-exact; only speed changes.                     */
int olv_autotune(olv_graph *g, const char *json_path, int reps);
int olv_autotune_load(olv_graph *g, const char *json_path, int *applied);

/* ---- traversal --------------------------------------------------------------
 * BFS levels: reproduces testBFS.cu:42-87 and BFS.cu:82-160 run to completion
 * (int32 level, 0x7fffffff unreached).  Direction-optimising (push/pull).      */
int olv_bfs(olv_graph *g, uint32_t src, int32_t *level_out, olv_stats *st);
/* BFS for callers that cannot allocate device memory (no reference
 * counterpart: the reference allocated in every VertexSubset and GRD).  The
 * caller passes the CSR (rowptr[V+1], col[E]) and level_out[V], all device
 * memory; nothing is allocated inside the call.  The engine's scratch is a
 * fixed file-scope device array (about 8.6 MB per GPU that loads the
 * library), so graphs are limited to 1,048,576 vertices and 16,777,216 edges
 * (larger ones return OLV_ERR_LIMIT).  Push-only traversal; the CSR is
 * validated on the device first.  The three arrays must be device memory of
 * the current device (or managed memory); anything else is OLV_ERR_ARG.  All
 * calls on a device share the scratch: calls that overlap on the GPU race.
 * The first call on a device looks up the scratch address and, under lazy
 * module loading, loads the library's device code there, which commits the
 * fixed scratch: make that call at initialisation time, before any stream
 * capture; later calls commit no memory.  st->device_ms is 0.               */
int olv_bfs_noalloc(const uint32_t *rowptr, const uint32_t *col, uint32_t V, uint64_t E,
                    uint32_t src, int32_t *level_out, void *stream, olv_stats *st);
/* SSSP distances with non-negative uint32 weights: the frontier Bellman-Ford of
 * SSSP.cu:106-174 (atomicMin relaxation) with near/far bucketing; a bucket's
 * heavy edges go by push or, where it reads fewer edges, by a pull over the
 * unsettled vertices' in-edges (tune key "sssp_pull").  uint32 distance,
 * 0x7fffffff unreached.  Needs an OLV_W_U32 graph.                             */
int olv_sssp(olv_graph *g, uint32_t src, uint32_t *dist_out, olv_stats *st);
/* Multi-source BFS (no reference counterpart): n <= 64 sources advanced
 * together with one 64-bit mask per vertex.  levels_out is [n][V] int32
 * (row s = BFS levels from srcs[s], 0x7fffffff unreached), each row equal to
 * olv_bfs from that source.  st->edges_traversed sums E_reached over sources. */
int olv_msbfs(olv_graph *g, const uint32_t *srcs, int n, int32_t *levels_out, olv_stats *st);
/* Batch of graphs packed block-diagonally (no reference counterpart).
 * olv_graph_create_er_batch builds `count` Erdos-Renyi digraphs, instance i
 * with V_i uniform in [vmin, vmax] and exactly avg_degree*V_i edges (no
 * self-loops or duplicates), packed in one CSR; inst_offsets[count+1]
 * receives the first global id of each instance.
 * olv_batch_run runs, in ONE persistent kernel with a device work queue, a
 * BFS from local vertex 0 of every instance (levels_out[V], levels relative
 * to the instance) and/or K <= 32 personalised PageRank vectors per instance
 * (seeds[count][K] local ids; ppr_out[V][K] FP32, vertex-major; dangling mass
 * returns to the seed; stop after max_it or when every vector's L1 change
 * < tol; ppr_iters_out[count] gets the iterations run).  Each instance's
 * result equals a run of that instance alone.  Instances hold <= 65,536
 * vertices.  Either output may be NULL.                                        */
int olv_graph_create_er_batch(int count, uint32_t vmin, uint32_t vmax, uint32_t avg_degree,
                              uint64_t seed, uint32_t *inst_offsets, olv_graph **out);
int olv_batch_run(olv_graph *g, const uint32_t *inst_offsets, int count, int K,
                  const uint32_t *seeds, double alpha, int max_it, double tol,
                  int32_t *levels_out, float *ppr_out, uint32_t *ppr_iters_out, olv_stats *st);
/* Differentiable weighted PageRank (no reference counterpart).  With
 * W_u = sum_v w_uv and P_uv = w_uv / W_u (rows without out-edges are zero):
 *   forward   r = (1-alpha) p + alpha P^T r           (pull over in-edges)
 *   backward  lambda = g + alpha P lambda             (pull over out-edges)
 *             dw_uv = alpha r_u (lambda_v - sum_x P_ux lambda_x) / W_u
 *             dp    = (1-alpha) lambda                for L = sum_v g_v r_v.
 * w (FP32, CSR order) replaces the graph's weights unless NULL (then the
 * graph must hold FP32 weights).  Each solve runs max_it Jacobi sweeps or
 * stops when the L1 change < tol.  *ctx is created on first use (pass a
 * pointer to NULL) and keeps r and W for the backward pass: O(V+E) memory, no
 * per-iteration tape.  dw_out is [E] in CSR order; dp_out may be NULL.       */
int olv_wpr_forward(olv_graph *g, const float *w, const float *p, double alpha, int max_it,
                    double tol, float *r_out, olv_wpr_ctx **ctx, olv_stats *st);
int olv_wpr_backward(olv_wpr_ctx *ctx, const float *g, int max_it, double tol, float *dw_out,
                     float *dp_out, olv_stats *st);
int olv_wpr_ctx_destroy(olv_wpr_ctx *ctx);
/* K personalised PageRank vectors on a general graph (no reference
 * counterpart; each vector follows PageRank.cu:51-75 with the teleport to its
 * own seed): for seed s_k, from r_k = e_{s_k},
 *   r_k'[v] = alpha * sum_{u->v} r_k[u]/outdeg(u) + [v == s_k]((1-alpha) + alpha d_k)
 * with d_k the vector's dangling mass (it returns to the seed).  K <= 32
 * vectors advance together: one pull over the reverse graph per iteration
 * gathers each in-neighbour's 128-byte row of K contributions (fixed order,
 * compensated FP32 sums; FP64 residual).  Stops after max_it iterations or
 * when every vector's L1 change < tol.  out is [V][K] FP32, vertex-major.  */
int olv_ppr_batch(olv_graph *g, const uint32_t *seeds, int K, double alpha, int max_it,
                  double tol, float *out, olv_stats *st);
/* PageRank (PageRank.cu:89-147 / testPageRank.cu:41-115), FP32 ranks from a
 * deterministic pull over the reverse graph, FP64 residual.  Runs max_it
 * iterations or until the L1 residual < tol.                                  */
int olv_pagerank(olv_graph *g, double alpha, int max_it, double tol, int dangling_mode,
                 float *rank_out, olv_stats *st);

/* ---- 1-D vertex partition (several GPUs) -----------------------------------
 * One rank's share of a graph split by contiguous vertex ranges (no working
 * reference counterpart: the reference's multi-GPU engine, olive.h:61-199 with
 * partition.h:95-436 and messageBox.h:66-105, never built).  The rank owns
 * vertices [lo, hi), lo a multiple of 64, and holds their in-edges: colptr
 * [hi-lo+1] (from 0) and rowidx (global source ids) of rows lo..hi-1 of the
 * reverse graph, and outdeg[hi-lo] (out-degrees in the whole graph).  The
 * exchange between ranks is the caller's (olive_b200/parallel.py: NCCL
 * all-gathers); the steps read replicated inputs and write the rank's slice.
 * Their array arguments are device memory.                                    */
typedef struct olv_part olv_part;
int olv_part_create(uint32_t V, uint32_t lo, uint32_t hi, const uint32_t *colptr,
                    const uint32_t *rowidx, const uint32_t *outdeg, olv_part **out);
int olv_part_destroy(olv_part *p);
int olv_part_set_stream(olv_part *p, void *stream);
/* BFS level L -> L+1, bottom-up over the owned vertices with level INT_MAX:
 * a vertex whose in-neighbour is set in frontier (V bits, 64-bit words) gets
 * level next_level and its bit in next (the owned words, bit i = vertex
 * lo + i; cleared first).  *found = vertices found.  Levels as testBFS.cu:64-79. */
int olv_part_bfs_step(olv_part *p, const uint64_t *frontier, int32_t *level, int32_t next_level,
                      uint64_t *next, uint64_t *found);
/* PageRank iteration over the owned rows (PageRank.cu:51-75 semantics):
 * rank[v] = base + alpha * sum_{u->v} contrib[u] (contrib = r/outdeg, all V),
 * contrib_out[v] = rank[v]/outdeg (0 for dangling vertices); sums[0] = sum of
 * |rank' - rank|, sums[1] = sum of the owned dangling ranks (FP64, host).    */
int olv_part_pr_step(olv_part *p, const float *contrib, double base, double alpha, float *rank,
                     float *contrib_out, double *sums);

/* ---- output ----------------------------------------------------------------
 * Write n values as text, one per line, byte for byte as the reference apps'
 * print() loops would (printVertices, oliver.h:204-212, with "%d\n" in
 * BFS.cu:41-43 / SSSP.cu:41-43 and "%f\n" in PageRank.cu:42-44, rounded as
 * glibc's printf rounds), formatted on the GPU in chunks of 2^24 values.
 * values may be host or device memory; stream is a cudaStream_t (NULL: the
 * default stream); *bytes_out (if not NULL) gets the file size.  "%f" values
 * of magnitude 2^107 or more return OLV_ERR_LIMIT.                           */
int olv_write_text(const char *path, const void *values, uint64_t n, int type, void *stream,
                   uint64_t *bytes_out);
/* Binary CSR dump (no reference counterpart): "OLVCSR1\n", uint64 V, E, flags
 * (bit 0: uint32 weights follow), uint32 rowptr[V+1], col[E], [weights[E]];
 * olv_graph_load reads it (either format value) and so does the header
 * layer's CsrGraph::fromEdgeListFile.                                         */
int olv_graph_save(const olv_graph *g, const char *path);

#ifdef __cplusplus
}
#endif
#endif /* OLIVE_B200_H */
