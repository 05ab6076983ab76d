"""CPU oracle for the olive_b200 frontier engine -- TEST INFRASTRUCTURE ONLY.

ctypes bindings for oracle/liboracle.so (the C restatement in oracle.c) plus
pure-Python restatements of the reference's graph loaders.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module,
and only as the checker: the product library never calls it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
INF = 0x7FFFFFFF

_lib = None


def build():
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        i32p = ctypes.POINTER(ctypes.c_int32)
        f64p = ctypes.POINTER(ctypes.c_double)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        c = ctypes
        L.orc_hash.restype = c.c_uint64
        L.orc_hash.argtypes = [c.c_uint64, c.c_uint64]
        L.orc_permute.restype = c.c_uint32
        L.orc_permute.argtypes = [c.c_uint32, c.c_int, c.c_uint64]
        L.orc_rmat_csr.restype = c.c_uint64
        L.orc_rmat_csr.argtypes = [c.c_int, c.c_int, c.c_uint64, u32p, u32p]
        L.orc_rmat_csr_par.restype = c.c_uint64
        L.orc_rmat_csr_par.argtypes = [c.c_int, c.c_int, c.c_uint64, c.c_int, u32p, u32p]
        L.orc_uint_weights_par.restype = None
        L.orc_uint_weights_par.argtypes = [c.c_uint64, c.c_uint64, c.c_uint32, c.c_uint32, u32p,
                                           c.c_int]
        L.orc_max_threads.restype = c.c_int
        L.orc_max_threads.argtypes = []
        L.orc_uint_weights.restype = None
        L.orc_uint_weights.argtypes = [c.c_uint64, c.c_uint64, c.c_uint32, c.c_uint32, u32p]
        L.orc_grid_csr.restype = c.c_uint64
        L.orc_grid_csr.argtypes = [c.c_uint32, c.c_uint32, u32p, u32p]
        L.orc_bfs.restype = c.c_uint64
        L.orc_bfs.argtypes = [c.c_uint32, u32p, u32p, c.c_uint32, i32p]
        L.orc_bfs_timed.restype = c.c_uint64
        L.orc_bfs_timed.argtypes = [c.c_uint32, u32p, u32p, c.c_uint32, i32p, c.c_double,
                                    f64p, u64p]
        L.orc_pagerank_leak.restype = c.c_int
        L.orc_pagerank_leak.argtypes = [c.c_uint32, u32p, u32p, c.c_int, f64p]
        L.orc_pagerank.restype = c.c_int
        L.orc_pagerank.argtypes = [c.c_uint32, u32p, u32p, c.c_double, c.c_int, c.c_double,
                                   f64p, f64p]
        L.orc_dijkstra.restype = c.c_uint64
        L.orc_dijkstra.argtypes = [c.c_uint32, u32p, u32p, u32p, c.c_uint32, u32p, c.c_double,
                                   f64p, u64p]
        L.orc_sssp_frontier.restype = c.c_uint64
        L.orc_sssp_frontier.argtypes = [c.c_uint32, u32p, u32p, u32p, c.c_uint32, u32p, c.c_int,
                                        c.c_double, f64p, u32p]
        L.orc_ppr.restype = c.c_int
        L.orc_ppr.argtypes = [c.c_uint32, u32p, u32p, c.c_int, u32p, c.c_double, c.c_int,
                              c.c_double, f64p]
        L.orc_sp_certificate.restype = c.c_uint64
        L.orc_sp_certificate.argtypes = [c.c_uint32, u32p, u32p, u32p, c.c_uint32, u32p, c.c_int,
                                         ctypes.POINTER(c.c_int)]
        L.orc_ppr_batch.restype = None
        L.orc_ppr_batch.argtypes = [c.c_int, u32p, u32p, u32p, c.c_int, u32p, c.c_double, c.c_int,
                                    i32p, c.c_double, f64p, i32p, c.c_int]
        L.orc_fprintf_i32.restype = c.c_double
        L.orc_fprintf_i32.argtypes = [c.c_char_p, i32p, c.c_uint64]
        L.orc_write_edge_list.restype = c.c_int
        L.orc_write_edge_list.argtypes = [c.c_char_p, c.c_uint32, u32p, u32p]
        L.orc_wpr_forward.restype = None
        L.orc_wpr_forward.argtypes = [c.c_uint32, u32p, u32p, f64p, f64p, c.c_double, c.c_int,
                                      f64p]
        L.orc_wpr_backward.restype = None
        L.orc_wpr_backward.argtypes = [c.c_uint32, u32p, u32p, f64p, f64p, f64p, c.c_double,
                                       c.c_int, f64p, f64p, f64p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


# --------------------------------------------------------------------------
# generators
# --------------------------------------------------------------------------
def rmat_csr(scale, ef=16, seed=1):
    V = 1 << scale
    rowptr = np.zeros(V + 1, np.uint32)
    col = np.zeros(ef * V, np.uint32)
    E = lib().orc_rmat_csr(scale, ef, seed, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32))
    return rowptr, col[:E].copy()


def rmat_csr_par(scale, ef=16, seed=1, threads=0):
    """orc_rmat_csr on all host threads (identical output)."""
    V = 1 << scale
    rowptr = np.zeros(V + 1, np.uint32)
    col = np.zeros(ef * V, np.uint32)
    E = lib().orc_rmat_csr_par(scale, ef, seed, threads, _p(rowptr, ctypes.c_uint32),
                               _p(col, ctypes.c_uint32))
    return rowptr, col[:E]


def uint_weights_par(E, seed, lo=1, hi=255, threads=0):
    w = np.zeros(max(E, 1), np.uint32)
    lib().orc_uint_weights_par(E, seed, lo, hi, _p(w, ctypes.c_uint32), threads)
    return w[:E]


def max_threads():
    return lib().orc_max_threads()


def uint_weights(E, seed, lo=1, hi=255):
    w = np.zeros(max(E, 1), np.uint32)
    lib().orc_uint_weights(E, seed, lo, hi, _p(w, ctypes.c_uint32))
    return w[:E]


_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _hash_np(seed, ctr):
    """orc_hash over a uint64 counter array (SplitMix64 output function of
    seed + ctr * golden ratio, arithmetic modulo 2^64)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.asarray(ctr, np.uint64) * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def er_instance(seed, n, m):
    """Edges (u, v) of one ER digraph of the batch generator
    (olive_b200/csrc/er_batch.cu; no reference counterpart): draw j gives
    (h(seed, 2j) mod n, h(seed, 2j+1) mod n); self-loops are dropped and the
    first m distinct pairs in draw order are kept, returned sorted by (u, v)."""
    m = min(int(m), n * (n - 1))
    draws = m + m // 4 + 64
    while True:
        j = np.arange(draws, dtype=np.uint64)
        u = _hash_np(seed, 2 * j) % np.uint64(n)
        v = _hash_np(seed, 2 * j + np.uint64(1)) % np.uint64(n)
        keep = u != v
        key = (u[keep] << np.uint64(32)) | v[keep]
        uniq, first = np.unique(key, return_index=True)
        if len(uniq) >= m or len(uniq) == n * (n - 1):
            chosen = np.sort(uniq[np.argsort(first, kind="stable")[:m]])
            return (chosen >> np.uint64(32)).astype(np.uint32), \
                (chosen & np.uint64(0xffffffff)).astype(np.uint32)
        draws *= 2


def er_batch_sizes(count, vmin, vmax, seed):
    """Vertex counts of the batch's instances (er_batch.cu er_instance_size)."""
    h = _hash_np(np.uint64(seed) ^ np.uint64(0xa5a5a5a5), np.arange(count, dtype=np.uint64))
    return (vmin + h % np.uint64(vmax - vmin + 1)).astype(np.int64)


def er_batch_instance(i, n, deg, seed):
    """Local CSR (rowptr, col) of instance i with n vertices."""
    s = int(_hash_np(seed, np.uint64(1000003 + i)))
    u, v = er_instance(s, n, deg * n)
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, u.astype(np.int64) + 1, 1)
    return np.cumsum(rp).astype(np.uint32), v


def grid_csr(rows, cols):
    V = rows * cols
    rowptr = np.zeros(V + 1, np.uint32)
    col = np.zeros(4 * V, np.uint32)
    E = lib().orc_grid_csr(rows, cols, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32))
    return rowptr, col[:E].copy()


# --------------------------------------------------------------------------
# algorithms
# --------------------------------------------------------------------------
def bfs(rowptr, col, src):
    rowptr, col = _u32(rowptr), _u32(col)
    V = len(rowptr) - 1
    level = np.empty(max(V, 1), np.int32)
    edges = lib().orc_bfs(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32), src,
                          _p(level, ctypes.c_int32))
    return level[:V], edges


def bfs_timed(rowptr, col, src, max_seconds):
    V = len(rowptr) - 1
    level = np.empty(V, np.int32)
    secs = ctypes.c_double()
    reached = ctypes.c_uint64()
    edges = lib().orc_bfs_timed(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32), src,
                                _p(level, ctypes.c_int32), max_seconds, ctypes.byref(secs),
                                ctypes.byref(reached))
    return edges, secs.value, reached.value


def pagerank_leak(rowptr, col, max_it=1000):
    rowptr, col = _u32(rowptr), _u32(col)
    V = len(rowptr) - 1
    r = np.empty(V, np.float64)
    it = lib().orc_pagerank_leak(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32),
                                 max_it, _p(r, ctypes.c_double))
    return r, it


def pagerank(rowptr, col, alpha=0.85, max_it=50, tol=1e-7):
    rowptr, col = _u32(rowptr), _u32(col)
    V = len(rowptr) - 1
    r = np.empty(V, np.float64)
    res = np.zeros(max(max_it, 1), np.float64)
    it = lib().orc_pagerank(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32), alpha,
                            max_it, tol, _p(r, ctypes.c_double), _p(res, ctypes.c_double))
    return r, it, res[:it]


def dijkstra(rowptr, col, w, src, max_seconds=0.0):
    rowptr, col, w = _u32(rowptr), _u32(col), _u32(w)
    V = len(rowptr) - 1
    dist = np.empty(max(V, 1), np.uint32)
    secs = ctypes.c_double()
    settled = ctypes.c_uint64()
    edges = lib().orc_dijkstra(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32),
                               _p(w, ctypes.c_uint32), src, _p(dist, ctypes.c_uint32),
                               max_seconds, ctypes.byref(secs), ctypes.byref(settled))
    return dist[:V], edges, secs.value, settled.value


def sssp_frontier(rowptr, col, w, src, threads=0, max_seconds=0.0):
    rowptr, col, w = _u32(rowptr), _u32(col), _u32(w)
    V = len(rowptr) - 1
    dist = np.empty(max(V, 1), np.uint32)
    secs = ctypes.c_double()
    rounds = ctypes.c_uint32()
    edges = lib().orc_sssp_frontier(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32),
                                    _p(w, ctypes.c_uint32), src, _p(dist, ctypes.c_uint32),
                                    threads, max_seconds, ctypes.byref(secs),
                                    ctypes.byref(rounds))
    return dist[:V], edges, secs.value, rounds.value


def ppr(rowptr, col, seeds, alpha=0.85, max_it=50, tol=1e-7):
    rowptr, col, seeds = _u32(rowptr), _u32(col), _u32(seeds)
    V = len(rowptr) - 1
    K = len(seeds)
    r = np.empty(V * K, np.float64)
    it = lib().orc_ppr(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32), K,
                       _p(seeds, ctypes.c_uint32), alpha, max_it, tol, _p(r, ctypes.c_double))
    return r.reshape(V, K), it


def sp_certificate(rowptr, col, dist, src, w=None, threads=0):
    """Check BFS levels (w None: unit weights) or SSSP distances by the
    shortest-path certificate of orc_sp_certificate.  Returns None when the
    certificate holds, else (vertex, reason)."""
    rowptr, col = _u32(rowptr), _u32(col)
    d = np.ascontiguousarray(dist).view(np.uint32) if np.asarray(dist).dtype.itemsize == 4 \
        else _u32(dist)
    V = len(rowptr) - 1
    wp = None if w is None else _p(_u32(w), ctypes.c_uint32)
    what = ctypes.c_int()
    r = lib().orc_sp_certificate(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32), wp,
                                 src, _p(d, ctypes.c_uint32), threads, ctypes.byref(what))
    if r == 0:
        return None
    return int(r - 1), {1: "source not at 0", 2: "edge not relaxed",
                        3: "no tight in-edge"}[what.value]


def ppr_batch(rowptr, col, inst_off, seeds, alpha=0.85, max_it=50, tol=1e-7, threads=0):
    """orc_ppr on every instance of a block-diagonal batch, instances in
    parallel: (r [V, K] FP64, iterations [count]).  max_it may be an array of
    per-instance iteration limits."""
    rowptr, col, off = _u32(rowptr), _u32(col), _u32(inst_off)
    seeds = _u32(seeds)
    count, K = seeds.shape
    V = int(off[-1])
    r = np.empty((V, K), np.float64)
    it = np.empty(count, np.int32)
    per = None
    if np.ndim(max_it):
        per = np.ascontiguousarray(max_it, np.int32)
        max_it = 0
    lib().orc_ppr_batch(count, _p(off, ctypes.c_uint32), _p(rowptr, ctypes.c_uint32),
                        _p(col, ctypes.c_uint32), K, _p(seeds, ctypes.c_uint32), alpha,
                        int(max_it), None if per is None else _p(per, ctypes.c_int32), tol,
                        _p(r, ctypes.c_double), _p(it, ctypes.c_int32), threads)
    return r, it


def wpr_forward(rowptr, col, w, p, alpha, iters):
    rowptr, col = _u32(rowptr), _u32(col)
    w = np.ascontiguousarray(w, np.float64)
    p = np.ascontiguousarray(p, np.float64)
    V = len(rowptr) - 1
    r = np.empty(V, np.float64)
    lib().orc_wpr_forward(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32),
                          _p(w, ctypes.c_double), _p(p, ctypes.c_double), alpha, iters,
                          _p(r, ctypes.c_double))
    return r


def wpr_backward(rowptr, col, w, r, g, alpha, iters):
    rowptr, col = _u32(rowptr), _u32(col)
    w = np.ascontiguousarray(w, np.float64)
    r = np.ascontiguousarray(r, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    V = len(rowptr) - 1
    lam = np.empty(V, np.float64)
    dw = np.empty(max(len(col), 1), np.float64)
    dp = np.empty(V, np.float64)
    lib().orc_wpr_backward(V, _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32),
                           _p(w, ctypes.c_double), _p(r, ctypes.c_double),
                           _p(g, ctypes.c_double), alpha, iters, _p(lam, ctypes.c_double),
                           _p(dw, ctypes.c_double), _p(dp, ctypes.c_double))
    return lam, dw[:len(col)], dp


# --------------------------------------------------------------------------
# the reference's loaders, restated
# --------------------------------------------------------------------------
def load_edge_list_ref(path):
    """CsrGraph::fromEdgeListFile as the reference executes it (csrGraph.h:106-171).

    Lines starting with '#' are skipped; the first other line is "V E"; each
    following line is "src dst [value]" and the value is ignored (:138-139).
    Rows are built assuming the tuples are grouped by source in increasing
    order (:149-165, the sort at :149 is commented out): an edge whose source
    is smaller than the previous one lands in the current row.  Returns
    (rowptr, col, weights-or-None) as uint32 arrays.
    """
    V = E = None
    src, dst, val = [], [], []
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            if not line or line[0] == "#":
                continue
            parts = line.split()
            if V is None:
                V, E = int(parts[0]), int(parts[1])
                continue
            src.append(int(parts[0]))
            dst.append(int(parts[1]))
            val.append(int(parts[2]) if len(parts) > 2 else None)
    rowptr = np.zeros(V + 1, np.int64)
    prev = -1
    for e in range(E):
        s = src[e]
        for v in range(prev + 1, s + 1):   # :151-157 "fill up the missing srcs"
            rowptr[v] = e
        prev = s
    for v in range(prev + 1, V + 1):       # :163-165 trailing vertices
        rowptr[v] = E
    col = np.asarray(dst[:E], np.uint32)
    w = None
    if E and all(x is not None for x in val):
        w = np.asarray(val[:E], np.uint32)
    return rowptr.astype(np.uint32), col, w


def load_edge_list_sorted(path):
    """The same file built into CSR with the tuples stably sorted by source
    (the evident intent of the commented-out sort at csrGraph.h:149)."""
    V = None
    src, dst, val = [], [], []
    with open(path) as f:
        for line in f:
            if not line.strip() or line[0] == "#":
                continue
            parts = line.split()
            if V is None:
                V = int(parts[0])
                continue
            src.append(int(parts[0]))
            dst.append(int(parts[1]))
            val.append(int(parts[2]) if len(parts) > 2 else 1)
    src = np.asarray(src, np.int64)
    order = np.argsort(src, kind="stable")
    rowptr = np.zeros(V + 1, np.int64)
    np.add.at(rowptr, src + 1, 1)
    rowptr = np.cumsum(rowptr)
    return (rowptr.astype(np.uint32), np.asarray(dst, np.uint32)[order],
            np.asarray(val, np.uint32)[order])


def fprintf_i32(path, values):
    """Write values with one fprintf("%d\\n") each (the reference's output
    loop); returns the seconds it took."""
    v = np.ascontiguousarray(values, np.int32)
    return lib().orc_fprintf_i32(str(path).encode(), _p(v, ctypes.c_int32), len(v))


def write_edge_list(path, rowptr, col, w=None):
    """Write CSR as a src-sorted edge-list file the reference loader reads."""
    if w is None:   # the C writer (fast at 10^8 edges)
        rowptr, col = _u32(rowptr), _u32(col)
        rc = lib().orc_write_edge_list(str(path).encode(), len(rowptr) - 1,
                                       _p(rowptr, ctypes.c_uint32), _p(col, ctypes.c_uint32))
        if rc != 0:
            raise OSError(f"cannot write {path}")
        return
    V = len(rowptr) - 1
    E = len(col)
    src = np.repeat(np.arange(V, dtype=np.int64), np.diff(rowptr.astype(np.int64)))
    with open(path, "w") as f:
        f.write("# olive_b200 edge list\n")
        f.write(f"{V} {E}\n")
        if w is None:
            np.savetxt(f, np.stack([src, col.astype(np.int64)], 1), fmt="%d")
        else:
            np.savetxt(f, np.stack([src, col.astype(np.int64), w.astype(np.int64)], 1),
                       fmt="%d")


def run_ref_bfs(path, src, workdir):
    """Run the reference's own testBFS (oracle/_ref) and read BFS.serial.txt."""
    exe = os.path.join(REF_DIR, "testBFS")
    out = subprocess.run([exe, path, "-s", str(src)], cwd=workdir, capture_output=True,
                         text=True, check=True)
    lv = np.loadtxt(os.path.join(workdir, "BFS.serial.txt"), dtype=np.int64, ndmin=1)
    return lv.astype(np.int32), out.stderr


def run_ref_pagerank(path, workdir, max_it=None):
    exe = os.path.join(REF_DIR, "testPageRank")
    cmd = [exe, path] + (["-max", str(max_it)] if max_it is not None else [])
    out = subprocess.run(cmd, cwd=workdir, capture_output=True, text=True, check=True)
    r = np.loadtxt(os.path.join(workdir, "PageRank.serial.txt"), dtype=np.float64, ndmin=1)
    return r, out.stderr
