/*
 * CPU oracle for the olive_b200 frontier engine.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the algorithms of
 * the reference's hot path (ACSAlab/olive) and the workload generators used by
 * the tests and the benchmark.  It is linked only by tests/, by the smoke check
 * in __graft_entry__.py and by bench.py's CPU-baseline leg, always as the
 * checker; the product path (libolive_b200.so) never calls it.
 *
 * Each routine cites the reference file:line it follows.  Routines with no
 * reference counterpart (Dijkstra, PageRank with dangling redistribution,
 * personalised PageRank, weighted PageRank and its adjoint, the generators)
 * say so and state the definition they implement.
 *
 * Pinning: orc_bfs and orc_pagerank_leak are checked against the unmodified
 * reference checkers (testBFS.cu, testPageRank.cu built from the reference
 * tree into oracle/_ref/) on every fixture in the reference's data/ directory,
 * on the 128x128 grid and on small RMAT graphs (tests/golden/).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_INF 0x7fffffff

static double orc_now(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* ------------------------------------------------------------------------ */
/* Counter-based random numbers: the SplitMix64 output function (Steele,   */
/* Lea, Flood 2014), applied to a counter.  The GPU generator in            */
/* olive_b200/csrc/graphgen.cu evaluates the same function, so both sides    */
/* draw identical graphs.                                                    */
/* ------------------------------------------------------------------------ */
#define ORC_GOLDEN 0x9E3779B97F4A7C15ULL

static inline uint64_t orc_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

uint64_t orc_hash(uint64_t seed, uint64_t ctr) {
    return orc_mix64(seed + ctr * ORC_GOLDEN);
}

/* Seeded bijection on [0, 2^bits): three rounds of (add, odd multiply,
 * xor-shift), each invertible modulo 2^bits. */
uint32_t orc_permute(uint32_t x, int bits, uint64_t seed) {
    uint64_t mask = (bits >= 64) ? ~0ULL : ((1ULL << bits) - 1);
    uint64_t y = x;
    int sh = (bits + 1) / 2;
    if (sh < 1) sh = 1;
    for (int r = 0; r < 3; r++) {
        uint64_t m = orc_hash(seed, 2 * r) | 1ULL;
        uint64_t c = orc_hash(seed, 2 * r + 1);
        y = (y + c) & mask;
        y = (y * m) & mask;
        y ^= (y >> sh);
        y &= mask;
    }
    return (uint32_t)y;
}

/* RMAT quadrant thresholds for (a,b,c,d) = (0.57,0.19,0.19,0.05) on a 32-bit
 * uniform draw: u < TA -> (0,0); u < TAB -> (0,1); u < TABC -> (1,0); else (1,1). */
#define ORC_TA   2448131359u   /* round(0.57 * 2^32) */
#define ORC_TAB  3264175145u   /* round(0.76 * 2^32) */
#define ORC_TABC 4080218931u   /* round(0.95 * 2^32) */

/* Raw RMAT draw of edge i (before permutation and clean-up). */
void orc_rmat_edge(int scale, uint64_t seed, uint64_t i, uint32_t *src, uint32_t *dst) {
    uint32_t s = 0, d = 0;
    for (int b = 0; b < scale; b++) {
        uint32_t u = (uint32_t)(orc_hash(seed, i * 64 + (uint64_t)b) >> 32);
        uint32_t sb, db;
        if (u < ORC_TA)        { sb = 0; db = 0; }
        else if (u < ORC_TAB)  { sb = 0; db = 1; }
        else if (u < ORC_TABC) { sb = 1; db = 0; }
        else                   { sb = 1; db = 1; }
        s = (s << 1) | sb;
        d = (d << 1) | db;
    }
    *src = s;
    *dst = d;
}

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

/*
 * RMAT graph (no reference counterpart): ef * 2^scale raw draws, ids permuted
 * by orc_permute(., scale, seed ^ perm_salt), self-loops dropped, duplicates
 * dropped, CSR sorted by (src, dst).  rowptr has 2^scale+1 entries; col must
 * hold ef * 2^scale entries.  Returns the edge count after clean-up.
 */
uint64_t orc_rmat_csr(int scale, int ef, uint64_t seed, uint32_t *rowptr, uint32_t *col) {
    uint64_t V = 1ULL << scale;
    uint64_t M = (uint64_t)ef * V;
    uint64_t *keys = (uint64_t *)malloc(M * sizeof(uint64_t));
    uint64_t n = 0;
    uint64_t pseed = seed ^ 0x5bd1e9955bd1e995ULL;
    for (uint64_t i = 0; i < M; i++) {
        uint32_t s, d;
        orc_rmat_edge(scale, seed, i, &s, &d);
        s = orc_permute(s, scale, pseed);
        d = orc_permute(d, scale, pseed);
        if (s == d) continue;
        keys[n++] = ((uint64_t)s << 32) | d;
    }
    qsort(keys, n, sizeof(uint64_t), cmp_u64);
    uint64_t m = 0;
    for (uint64_t i = 0; i < n; i++)
        if (i == 0 || keys[i] != keys[i - 1]) keys[m++] = keys[i];
    memset(rowptr, 0, (V + 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < m; i++) {
        rowptr[(keys[i] >> 32) + 1]++;
        col[i] = (uint32_t)keys[i];
    }
    for (uint64_t v = 0; v < V; v++) rowptr[v + 1] += rowptr[v];
    free(keys);
    return m;
}

/* Edge weights in [lo, hi], drawn from the stream indexed by CSR position. */
void orc_uint_weights(uint64_t E, uint64_t seed, uint32_t lo, uint32_t hi, uint32_t *w) {
    uint32_t span = hi - lo + 1;
    for (uint64_t e = 0; e < E; e++)
        w[e] = lo + (uint32_t)((orc_hash(seed, e) >> 32) % span);
}

/* 2-D grid, 4-neighbour, both directions, id = r*cols + c, neighbours in
 * (up, left, right, down) order.  Returns E. */
uint64_t orc_grid_csr(uint32_t rows, uint32_t cols, uint32_t *rowptr, uint32_t *col) {
    uint64_t e = 0;
    for (uint32_t r = 0; r < rows; r++)
        for (uint32_t c = 0; c < cols; c++) {
            uint32_t v = r * cols + c;
            rowptr[v] = (uint32_t)e;
            if (r > 0) col[e++] = v - cols;
            if (c > 0) col[e++] = v - 1;
            if (c + 1 < cols) col[e++] = v + 1;
            if (r + 1 < rows) col[e++] = v + cols;
        }
    rowptr[(uint64_t)rows * cols] = (uint32_t)e;
    return e;
}

/* ------------------------------------------------------------------------ */
/* BFS: testBFS.cu:56-79 (CLRS queue BFS; INT_MAX = 0x7fffffff unreached).  */
/* ------------------------------------------------------------------------ */
uint64_t orc_bfs(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                 uint32_t src, int32_t *level) {
    for (uint32_t i = 0; i < V; i++) level[i] = ORC_INF;   /* testBFS.cu:56-59 */
    if (V == 0) return 0;
    level[src] = 0;                                         /* testBFS.cu:60 */
    uint32_t *q = (uint32_t *)malloc((size_t)V * sizeof(uint32_t));
    size_t head = 0, tail = 0;
    q[tail++] = src;
    uint64_t edges = 0;
    while (head < tail) {                                   /* testBFS.cu:67-79 */
        uint32_t v = q[head++];
        for (uint32_t e = rowptr[v]; e < rowptr[v + 1]; e++) {
            uint32_t d = col[e];
            if (level[d] == ORC_INF) {
                level[d] = level[v] + 1;
                q[tail++] = d;
            }
        }
        edges += rowptr[v + 1] - rowptr[v];
    }
    free(q);
    return edges;   /* sum of out-degrees of reached vertices */
}

/* Bounded BFS for the timed CPU baseline: stops after max_seconds.
 * Returns edges scanned; *reached receives dequeued vertices. */
uint64_t orc_bfs_timed(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                       uint32_t src, int32_t *level, double max_seconds,
                       double *seconds, uint64_t *reached) {
    for (uint32_t i = 0; i < V; i++) level[i] = ORC_INF;
    uint32_t *q = (uint32_t *)malloc((size_t)V * sizeof(uint32_t));
    double t0 = orc_now();
    size_t head = 0, tail = 0;
    level[src] = 0;
    q[tail++] = src;
    uint64_t edges = 0;
    while (head < tail) {
        uint32_t v = q[head++];
        for (uint32_t e = rowptr[v]; e < rowptr[v + 1]; e++) {
            uint32_t d = col[e];
            if (level[d] == ORC_INF) {
                level[d] = level[v] + 1;
                q[tail++] = d;
            }
        }
        edges += rowptr[v + 1] - rowptr[v];
        if ((head & 0xffff) == 0 && orc_now() - t0 > max_seconds) break;
    }
    *seconds = orc_now() - t0;
    *reached = head;
    free(q);
    return edges;
}

/* ------------------------------------------------------------------------ */
/* PageRank exactly as testPageRank.cu:57-104: FP64 push over CSR, dangling */
/* mass leaks, stop when sum|delta| < 1e-7 or after max_it iterations.      */
/* Returns the iteration counter the reference prints.                      */
/* ------------------------------------------------------------------------ */
int orc_pagerank_leak(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                      int max_it, double *ranks) {
    const double damping = 0.85;                          /* testPageRank.cu:57 */
    const double oneOverN = 1.0 / V;
    const double epsilon = 0.0000001;
    double *deltas = (double *)malloc((size_t)V * sizeof(double));
    double *ngh = (double *)malloc((size_t)V * sizeof(double));
    for (uint32_t i = 0; i < V; i++) { ranks[i] = oneOverN; deltas[i] = oneOverN; ngh[i] = 0; }
    int iterations = 0;
    while (iterations < max_it) {                         /* testPageRank.cu:74 */
        for (uint32_t i = 0; i < V; i++) ngh[i] = 0;
        for (uint32_t v = 0; v < V; v++)                  /* :79-85 */
            for (uint32_t e = rowptr[v]; e < rowptr[v + 1]; e++) {
                uint32_t outdeg = rowptr[v + 1] - rowptr[v];
                ngh[col[e]] += ranks[v] / outdeg;
            }
        for (uint32_t v = 0; v < V; v++) {                /* :87-91 */
            double nr = damping * ngh[v] + (1 - damping) * oneOverN;
            deltas[v] = nr - ranks[v];
            ranks[v] = nr;
        }
        double err = 0.0;                                 /* :93-96 */
        for (uint32_t i = 0; i < V; i++) err += fabs(deltas[i]);
        if (err < epsilon) break;                         /* :102 */
        iterations++;
    }
    free(deltas);
    free(ngh);
    return iterations;
}

/*
 * PageRank with uniform dangling redistribution (no reference counterpart;
 * the reference leaks dangling mass).  FP64.  Each iteration:
 *   d = sum of r[u] over out-degree-0 u
 *   r'[v] = (1-alpha)/N + alpha * (sum_{u->v} r[u]/outdeg(u) + d/N)
 *   res = sum |r' - r|;  r = r';  stop after max_it or when res < tol.
 * Returns iterations performed; residuals[i] (if non-NULL) gets res of i.
 */
int orc_pagerank(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                 double alpha, int max_it, double tol, double *r, double *residuals) {
    double *s = (double *)malloc((size_t)V * sizeof(double));
    for (uint32_t v = 0; v < V; v++) r[v] = 1.0 / V;
    int it = 0;
    while (it < max_it) {
        double d = 0.0;
        for (uint32_t v = 0; v < V; v++) {
            s[v] = 0.0;
            if (rowptr[v + 1] == rowptr[v]) d += r[v];
        }
        for (uint32_t u = 0; u < V; u++) {
            uint32_t deg = rowptr[u + 1] - rowptr[u];
            if (!deg) continue;
            double c = r[u] / deg;
            for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) s[col[e]] += c;
        }
        double base = (1.0 - alpha) / V + alpha * d / V;
        double res = 0.0;
        for (uint32_t v = 0; v < V; v++) {
            double nr = base + alpha * s[v];
            res += fabs(nr - r[v]);
            r[v] = nr;
        }
        if (residuals) residuals[it] = res;
        it++;
        if (res < tol) break;
    }
    free(s);
    return it;
}

/* ------------------------------------------------------------------------ */
/* SSSP                                                                      */
/* ------------------------------------------------------------------------ */
typedef struct { uint32_t d, v; } orc_hitem;

static void heap_push(orc_hitem *h, size_t *n, orc_hitem x) {
    size_t i = (*n)++;
    while (i > 0) {
        size_t p = (i - 1) >> 1;
        if (h[p].d <= x.d) break;
        h[i] = h[p];
        i = p;
    }
    h[i] = x;
}

static orc_hitem heap_pop(orc_hitem *h, size_t *n) {
    orc_hitem top = h[0];
    orc_hitem x = h[--(*n)];
    size_t i = 0;
    for (;;) {
        size_t c = 2 * i + 1;
        if (c >= *n) break;
        if (c + 1 < *n && h[c + 1].d < h[c].d) c++;
        if (h[c].d >= x.d) break;
        h[i] = h[c];
        i = c;
    }
    h[i] = x;
    return top;
}

/*
 * Serial Dijkstra with a binary heap and lazy deletion (no reference
 * counterpart: the reference has no SSSP checker).  uint32 distances,
 * 0x7fffffff = unreached (the reference SSSP's infDistance, SSSP.cu:123).
 * Stops early after max_seconds (<= 0: no limit).  Returns edges scanned
 * (sum of out-degrees of settled vertices); *settled gets their count.
 */
uint64_t orc_dijkstra(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                      const uint32_t *w, uint32_t src, uint32_t *dist,
                      double max_seconds, double *seconds, uint64_t *settled) {
    for (uint32_t v = 0; v < V; v++) dist[v] = ORC_INF;
    uint8_t *done = (uint8_t *)calloc(V ? V : 1, 1);
    size_t cap = (size_t)rowptr[V] + 2, n = 0;
    orc_hitem *h = (orc_hitem *)malloc(cap * sizeof(orc_hitem));
    double t0 = orc_now();
    uint64_t edges = 0, nset = 0;
    if (V) {
        dist[src] = 0;
        orc_hitem s0 = {0, src};
        heap_push(h, &n, s0);
    }
    while (n) {
        orc_hitem it = heap_pop(h, &n);
        if (done[it.v]) continue;
        done[it.v] = 1;
        nset++;
        uint32_t du = it.d;
        for (uint32_t e = rowptr[it.v]; e < rowptr[it.v + 1]; e++) {
            uint32_t v = col[e];
            uint32_t nd = du + w[e];
            if (nd < dist[v]) {
                dist[v] = nd;
                orc_hitem x = {nd, v};
                heap_push(h, &n, x);
            }
        }
        edges += rowptr[it.v + 1] - rowptr[it.v];
        if (max_seconds > 0 && (nset & 0xffff) == 0 && orc_now() - t0 > max_seconds) break;
    }
    if (seconds) *seconds = orc_now() - t0;
    if (settled) *settled = nset;
    free(h);
    free(done);
    return edges;
}

/*
 * Frontier Bellman-Ford in the reference's superstep form (SSSP.cu:146-163
 * driving Oliver::edgeFilter / vertexFilter, oliver.h:56-113, kernels
 * oliverKernel.h:45-141):
 *   edgeFilter:  acc[*] = INF (oliver.h:66); for u in queue, for each edge:
 *                acc[v] = min(acc[v], dist[u] + w) (SSSP.cu:54-64); flag[v] = 1
 *   vertexFilter: for flagged v with dist[v] > acc[v] (SSSP.cu:72-75, with the
 *                accumulator passed to cond): dist[v] = acc[v]; enqueue v
 * until the queue is empty.  Weights are the given ones (the reference app
 * forces them to 1, SSSP.cu:131).  Runs on nthreads OpenMP threads with an
 * atomic minimum.  Stops after max_seconds (<= 0: no limit).  Returns edges
 * scanned; *rounds gets the superstep count.
 */
uint64_t orc_sssp_frontier(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                           const uint32_t *w, uint32_t src, uint32_t *dist,
                           int nthreads, double max_seconds, double *seconds,
                           uint32_t *rounds) {
    uint32_t *acc = (uint32_t *)malloc((size_t)V * sizeof(uint32_t));
    uint8_t *flag = (uint8_t *)malloc(V ? V : 1);
    uint32_t *q = (uint32_t *)malloc((size_t)V * sizeof(uint32_t));
    uint32_t *nq = (uint32_t *)malloc((size_t)V * sizeof(uint32_t));
    uint64_t qn = 0, edges = 0;
    uint32_t nr = 0;
    double t0 = orc_now();
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    for (uint32_t v = 0; v < V; v++) dist[v] = ORC_INF;
    if (V) { dist[src] = 0; q[qn++] = src; }
    while (qn) {
        #pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < (int64_t)V; v++) { acc[v] = ORC_INF; flag[v] = 0; }
        uint64_t scanned = 0;
        #pragma omp parallel for schedule(dynamic, 64) reduction(+:scanned)
        for (int64_t i = 0; i < (int64_t)qn; i++) {
            uint32_t u = q[i];
            uint32_t du = dist[u];
            for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) {
                uint32_t v = col[e];
                uint32_t nd = du + w[e];
                uint32_t cur = __atomic_load_n(&acc[v], __ATOMIC_RELAXED);
                while (nd < cur &&
                       !__atomic_compare_exchange_n(&acc[v], &cur, nd, 1,
                                                    __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
                flag[v] = 1;
            }
            scanned += rowptr[u + 1] - rowptr[u];
        }
        edges += scanned;
        uint64_t nn = 0;
        #pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < (int64_t)V; v++) {
            if (flag[v] && dist[v] > acc[v]) {
                dist[v] = acc[v];
                uint64_t pos = __atomic_fetch_add(&nn, 1, __ATOMIC_RELAXED);
                nq[pos] = (uint32_t)v;
            }
        }
        uint32_t *t = q; q = nq; nq = t;
        qn = nn;
        nr++;
        if (max_seconds > 0 && orc_now() - t0 > max_seconds) break;
    }
    if (seconds) *seconds = orc_now() - t0;
    if (rounds) *rounds = nr;
    free(acc); free(flag); free(q); free(nq);
    return edges;
}

/* ------------------------------------------------------------------------ */
/* Personalised PageRank, K vectors (no reference counterpart).  FP64.      */
/* For seed s_k:  r_k'[v] = (1-alpha)[v==s_k]                                */
/*                        + alpha * (sum_{u->v} r_k[u]/outdeg(u) + d_k[v==s_k]) */
/* with d_k the dangling mass of r_k; r_k starts one-hot at s_k.  Stops     */
/* after max_it iterations or when max_k sum|r_k' - r_k| < tol.  Output is   */
/* vertex-major: r[v*K + k].  Returns iterations performed.                   */
/* ------------------------------------------------------------------------ */
int orc_ppr(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
            int K, const uint32_t *seeds, double alpha, int max_it, double tol, double *r) {
    size_t n = (size_t)V * K;
    double *s = (double *)malloc(n * sizeof(double));
    double *d = (double *)malloc(K * sizeof(double));
    double *res = (double *)malloc(K * sizeof(double));
    memset(r, 0, n * sizeof(double));
    for (int k = 0; k < K; k++) r[(size_t)seeds[k] * K + k] = 1.0;
    int it = 0;
    while (it < max_it) {
        memset(s, 0, n * sizeof(double));
        for (int k = 0; k < K; k++) { d[k] = 0; res[k] = 0; }
        for (uint32_t u = 0; u < V; u++) {
            uint32_t deg = rowptr[u + 1] - rowptr[u];
            if (!deg) {
                for (int k = 0; k < K; k++) d[k] += r[(size_t)u * K + k];
                continue;
            }
            for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++)
                for (int k = 0; k < K; k++)
                    s[(size_t)col[e] * K + k] += r[(size_t)u * K + k] / deg;
        }
        for (uint32_t v = 0; v < V; v++)
            for (int k = 0; k < K; k++) {
                double t = (seeds[k] == v) ? (1.0 - alpha) + alpha * d[k] : 0.0;
                double nv = t + alpha * s[(size_t)v * K + k];
                res[k] += fabs(nv - r[(size_t)v * K + k]);
                r[(size_t)v * K + k] = nv;
            }
        it++;
        double mx = 0;
        for (int k = 0; k < K; k++) if (res[k] > mx) mx = res[k];
        if (mx < tol) break;
    }
    free(s); free(d); free(res);
    return it;
}

/* ------------------------------------------------------------------------ */
/* Weighted PageRank and its adjoint (no reference counterpart).  FP64.     */
/*   W_u = sum_v w_uv,  P_uv = w_uv / W_u  (rows with no out-edges are 0)    */
/*   forward:  r = (1-alpha) p + alpha P^T r                                  */
/*   adjoint:  lambda = g + alpha P lambda                                    */
/*   dL/dw_uv = alpha r_u (lambda_v - sum_x P_ux lambda_x) / W_u              */
/*   dL/dp    = (1-alpha) lambda                                              */
/* Both solves are Jacobi iterations from r = p (resp. lambda = g) run for   */
/* exactly `iters` sweeps.                                                    */
/* ------------------------------------------------------------------------ */
void orc_wpr_forward(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                     const double *w, const double *p, double alpha, int iters, double *r) {
    double *W = (double *)malloc((size_t)V * sizeof(double));
    double *s = (double *)malloc((size_t)V * sizeof(double));
    for (uint32_t u = 0; u < V; u++) {
        double t = 0;
        for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) t += w[e];
        W[u] = t;
        r[u] = p[u];
    }
    for (int it = 0; it < iters; it++) {
        for (uint32_t v = 0; v < V; v++) s[v] = 0;
        for (uint32_t u = 0; u < V; u++) {
            if (rowptr[u + 1] == rowptr[u]) continue;
            double ru = r[u] / W[u];
            for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) s[col[e]] += w[e] * ru;
        }
        for (uint32_t v = 0; v < V; v++) r[v] = (1 - alpha) * p[v] + alpha * s[v];
    }
    free(W); free(s);
}

void orc_wpr_backward(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                      const double *w, const double *r, const double *g, double alpha,
                      int iters, double *lam, double *dw, double *dp) {
    double *W = (double *)malloc((size_t)V * sizeof(double));
    double *t = (double *)malloc((size_t)V * sizeof(double));
    for (uint32_t u = 0; u < V; u++) {
        double x = 0;
        for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) x += w[e];
        W[u] = x;
        lam[u] = g[u];
    }
    for (int it = 0; it < iters; it++) {
        for (uint32_t u = 0; u < V; u++) {
            double x = 0;
            if (W[u] != 0)
                for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) x += w[e] * lam[col[e]];
            t[u] = (W[u] != 0) ? x / W[u] : 0.0;
        }
        for (uint32_t u = 0; u < V; u++) lam[u] = g[u] + alpha * t[u];
    }
    for (uint32_t u = 0; u < V; u++) {
        double x = 0;
        if (W[u] != 0)
            for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) x += w[e] * lam[col[e]];
        t[u] = (W[u] != 0) ? x / W[u] : 0.0;
    }
    for (uint32_t u = 0; u < V; u++) {
        for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++)
            dw[e] = alpha * r[u] * (lam[col[e]] - t[u]) / W[u];
        dp[u] = (1 - alpha) * lam[u];
    }
    free(W); free(t);
}

/* ------------------------------------------------------------------------ */
/* Parallel host version of orc_rmat_csr (same graph, bit for bit): OpenMP */
/* key generation and an LSD radix sort over the 2*scale significant bits.  */
/* Used to build the benchmark graph on the host for the CPU reference arm. */
/* ------------------------------------------------------------------------ */
static void radix_sort_u64(uint64_t *a, uint64_t *tmp, uint64_t n, int bits, int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    const int R = 256;
    size_t *hist = (size_t *)calloc((size_t)nthreads * R, sizeof(size_t));
    for (int shift = 0; shift < bits; shift += 8) {
        memset(hist, 0, (size_t)nthreads * R * sizeof(size_t));
        #pragma omp parallel num_threads(nthreads)
        {
#ifdef _OPENMP
            int t = omp_get_thread_num();
#else
            int t = 0;
#endif
            uint64_t lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
            size_t *h = hist + (size_t)t * R;
            for (uint64_t i = lo; i < hi; i++) h[(a[i] >> shift) & 255]++;
            #pragma omp barrier
            #pragma omp single
            {
                size_t sum = 0;
                for (int d = 0; d < R; d++)
                    for (int tt = 0; tt < nthreads; tt++) {
                        size_t c = hist[(size_t)tt * R + d];
                        hist[(size_t)tt * R + d] = sum;
                        sum += c;
                    }
            }
            for (uint64_t i = lo; i < hi; i++) tmp[h[(a[i] >> shift) & 255]++] = a[i];
        }
        memcpy(a, tmp, n * sizeof(uint64_t));
    }
    free(hist);
}

uint64_t orc_rmat_csr_par(int scale, int ef, uint64_t seed, int nthreads, uint32_t *rowptr,
                          uint32_t *col) {
    uint64_t V = 1ULL << scale;
    uint64_t M = (uint64_t)ef * V;
    uint64_t *keys = (uint64_t *)malloc(M * sizeof(uint64_t));
    uint64_t *tmp = (uint64_t *)malloc(M * sizeof(uint64_t));
    uint64_t pseed = seed ^ 0x5bd1e9955bd1e995ULL;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    #pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < (int64_t)M; i++) {
        uint32_t s, d;
        orc_rmat_edge(scale, seed, (uint64_t)i, &s, &d);
        s = orc_permute(s, scale, pseed);
        d = orc_permute(d, scale, pseed);
        /* compact key (s << scale | d); a self-loop becomes all ones (sorted last) */
        keys[i] = (s == d) ? ~0ULL : (((uint64_t)s << scale) | d);
    }
    radix_sort_u64(keys, tmp, M, 2 * scale, nthreads);
    free(tmp);
    uint64_t m = 0;
    const uint64_t dmask = V - 1;
    memset(rowptr, 0, (V + 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < M; i++) {
        if (keys[i] == ~0ULL) break;
        if (i && keys[i] == keys[i - 1]) continue;
        rowptr[(keys[i] >> scale) + 1]++;
        col[m++] = (uint32_t)(keys[i] & dmask);
    }
    for (uint64_t v = 0; v < V; v++) rowptr[v + 1] += rowptr[v];
    free(keys);
    return m;
}

void orc_uint_weights_par(uint64_t E, uint64_t seed, uint32_t lo, uint32_t hi, uint32_t *w,
                          int nthreads) {
    uint32_t span = hi - lo + 1;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    #pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t e = 0; e < (int64_t)E; e++)
        w[e] = lo + (uint32_t)((orc_hash(seed, (uint64_t)e) >> 32) % span);
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Shortest-path certificate (no reference counterpart; the size-independent */
/* check used where a full serial oracle run is too slow).  For BFS levels    */
/* (w == NULL: every edge weighs 1) or SSSP distances (weights >= 1):         */
/*   d[src] == 0, every reached vertex other than src has d > 0;              */
/*   every edge (u,v) with u reached satisfies d[v] <= d[u] + w(u,v);         */
/*   every reached v != src has a tight in-edge: d[v] == d[u] + w(u,v).       */
/* With strictly positive weights these conditions hold for the exact         */
/* distances and for nothing else (tight edges strictly decrease d, so they   */
/* lead back to src; the edge condition bounds d from below).  Unreached     */
/* vertices (0x7fffffff) may have no reached in-neighbour, which the edge     */
/* condition enforces.  Returns 0 when valid, else 1 + the offending vertex   */
/* (an edge violation reports its target) with *what = 1 (source), 2 (edge),  */
/* 3 (no tight in-edge).                                                      */
/* ------------------------------------------------------------------------ */
uint64_t orc_sp_certificate(uint32_t V, const uint32_t *rowptr, const uint32_t *col,
                            const uint32_t *w, uint32_t src, const uint32_t *d,
                            int nthreads, int *what) {
    *what = 0;
    if (V == 0) return 0;
    if (d[src] != 0) { *what = 1; return (uint64_t)src + 1; }
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    uint8_t *tight = (uint8_t *)calloc(V, 1);
    uint64_t bad = 0;
    #pragma omp parallel for schedule(dynamic, 4096) num_threads(nthreads)
    for (int64_t u = 0; u < (int64_t)V; u++) {
        const uint64_t du = d[u];
        if (du == ORC_INF) continue;
        for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) {
            const uint32_t v = col[e];
            const uint64_t nd = du + (w ? w[e] : 1u);
            if ((uint64_t)d[v] > nd) {
                uint64_t z = 0;
                __atomic_compare_exchange_n(&bad, &z, (uint64_t)v + 1, 0, __ATOMIC_RELAXED,
                                            __ATOMIC_RELAXED);
            } else if ((uint64_t)d[v] == nd) {
                __atomic_store_n(&tight[v], (uint8_t)1, __ATOMIC_RELAXED);
            }
        }
    }
    if (bad) { free(tight); *what = 2; return bad; }
    for (uint32_t v = 0; v < V; v++)
        if (v != src && d[v] != ORC_INF && (d[v] == 0 || !tight[v])) {
            free(tight);
            *what = 3;
            return (uint64_t)v + 1;
        }
    free(tight);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* orc_ppr over every instance of a block-diagonal batch (instances run in   */
/* parallel on the host threads, each one exactly as orc_ppr runs it alone).  */
/* inst_off[count+1] are the first global ids; seeds[count][K] local ids;     */
/* instance i runs at most max_its[i] iterations (max_it when max_its is      */
/* NULL); r[V][K] receives each instance's vectors at its global rows;        */
/* iters[count] the iterations each ran.                                      */
/* ------------------------------------------------------------------------ */
void orc_ppr_batch(int count, const uint32_t *inst_off, const uint32_t *rowptr,
                   const uint32_t *col, int K, const uint32_t *seeds, double alpha, int max_it,
                   const int32_t *max_its, double tol, double *r, int32_t *iters,
                   int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    #pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int i = 0; i < count; i++) {
        const uint32_t b = inst_off[i], n = inst_off[i + 1] - b;
        const uint32_t e0 = rowptr[b], m = rowptr[b + n] - e0;
        uint32_t *lrp = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
        uint32_t *lcl = (uint32_t *)malloc(((size_t)m + 1) * sizeof(uint32_t));
        for (uint32_t v = 0; v <= n; v++) lrp[v] = rowptr[b + v] - e0;
        for (uint32_t e = 0; e < m; e++) lcl[e] = col[e0 + e] - b;
        iters[i] = orc_ppr(n, lrp, lcl, K, seeds + (size_t)i * K, alpha,
                           max_its ? max_its[i] : max_it, tol, r + (size_t)b * K);
        free(lrp);
        free(lcl);
    }
}

/* ------------------------------------------------------------------------ */
/* Write a CSR as the text edge list CsrGraph::fromEdgeListFile reads        */
/* (csrGraph.h:106-171): a '#' comment line, "V E", then "src dst" per edge   */
/* in CSR order (sorted by source, as that loader requires).  Returns 0, or  */
/* -1 when the file cannot be written.  Used to run the reference's own      */
/* testBFS / testPageRank binaries on the benchmark graphs.                   */
/* ------------------------------------------------------------------------ */
static char *orc_utoa(char *p, uint64_t x) {
    char t[24];
    int n = 0;
    do { t[n++] = (char)('0' + x % 10); x /= 10; } while (x);
    while (n) *p++ = t[--n];
    return p;
}

int orc_write_edge_list(const char *path, uint32_t V, const uint32_t *rowptr,
                        const uint32_t *col) {
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    const uint64_t E = rowptr[V];
    fprintf(f, "# olive_b200 edge list\n%u %llu\n", V, (unsigned long long)E);
    const size_t cap = 1 << 22;
    char *buf = (char *)malloc(cap + 64);
    size_t n = 0;
    for (uint32_t u = 0; u < V; u++)
        for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) {
            char *p = buf + n;
            p = orc_utoa(p, u);
            *p++ = ' ';
            p = orc_utoa(p, col[e]);
            *p++ = '\n';
            n = (size_t)(p - buf);
            if (n >= cap) {
                if (fwrite(buf, 1, n, f) != n) { free(buf); fclose(f); return -1; }
                n = 0;
            }
        }
    int rc = (n && fwrite(buf, 1, n, f) != n) ? -1 : 0;
    free(buf);
    if (fclose(f) != 0) rc = -1;
    return rc;
}

/* ------------------------------------------------------------------------ */
/* The reference's way of writing results: one fprintf("%d\n") per vertex    */
/* on the host (printVertices, oliver.h:204-212, through BFS_Vertex::print,  */
/* BFS.cu:41-43).  Baseline for the GPU writer; returns seconds, < 0 when    */
/* the file cannot be written.                                                */
/* ------------------------------------------------------------------------ */
double orc_fprintf_i32(const char *path, const int32_t *v, uint64_t n) {
    double t0 = orc_now();
    FILE *f = fopen(path, "w");
    if (!f) return -1.0;
    for (uint64_t i = 0; i < n; i++) fprintf(f, "%d\n", v[i]);
    if (fclose(f) != 0) return -1.0;
    return orc_now() - t0;
}
