"""olive_b200 -- a B200-native frontier graph engine (ACSAlab/olive semantics).

Python view of the C ABI in include/olive_b200.h (libolive_b200.so, loaded
with ctypes).  Arrays may be numpy arrays (host) or CUDA torch tensors
(device); outputs land where the `out` argument lives, or in a new numpy array.
There is no CPU fallback: if the library is missing or a call fails, an
exception is raised.
"""
import ctypes
import os

import numpy as np

__all__ = ["Graph", "OliveError", "lib", "INF", "Stats", "write_csr_binary", "write_text"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libolive_b200.so")
INF = 0x7FFFFFFF

W_NONE, W_U32, W_F32 = 0, 1, 2
DANGLING = {"uniform": 0, "leak": 1}


class OliveError(RuntimeError):
    pass


CSR_MAGIC = b"OLVCSR1\n"


def write_csr_binary(path, rowptr, col, values=None):
    """Write a binary CSR dump that CsrGraph::fromEdgeListFile (include/olive/
    csrGraph.h) and olv_graph_load read: "OLVCSR1\\n", uint64 V, E, flags
    (bit 0: uint32 edge values follow), uint32 rowptr[V+1], col[E], [values]."""
    rowptr = np.ascontiguousarray(rowptr, np.uint32)
    col = np.ascontiguousarray(col, np.uint32)
    V, E = len(rowptr) - 1, len(col)
    with open(path, "wb") as f:
        f.write(CSR_MAGIC)
        f.write(np.array([V, E, 0 if values is None else 1], np.uint64).tobytes())
        rowptr.tofile(f)
        col.tofile(f)
        if values is not None:
            np.ascontiguousarray(values, np.uint32).tofile(f)


def write_text(path, values, stream=None):
    """Write values (int32 -> "%d", uint32 -> "%u", float32/float64 -> "%f"),
    one per line, formatted on the GPU (olv_write_text).  values: a numpy
    array or a CUDA tensor.  Returns the bytes written."""
    dt = str(values.dtype).replace("torch.", "")
    if dt not in TEXT_TYPES:
        raise ValueError(f"write_text: unsupported dtype {values.dtype}")
    n = values.numel() if hasattr(values, "numel") else values.size
    out = _U64()
    s = getattr(stream, "cuda_stream", stream)
    _check(lib().olv_write_text(str(path).encode(), _ptr(values), n, TEXT_TYPES[dt], s,
                                ctypes.byref(out)), "olv_write_text")
    return out.value


class Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint32), ("pull_steps", ctypes.c_uint32),
                ("vertices_reached", ctypes.c_uint64), ("edges_traversed", ctypes.c_uint64),
                ("edges_relaxed", ctypes.c_uint64), ("residual", ctypes.c_double),
                ("device_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

# (name, restype, argtypes) of every entry point in include/olive_b200.h
_VP = ctypes.c_void_p
_U32, _U64, _I, _D = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
_SIGS = [
    ("olv_last_error", ctypes.c_char_p, []),
    ("olv_version", ctypes.c_char_p, []),
    ("olv_graph_create", _I, [_VP, _VP, _VP, _I, _U32, _U64, ctypes.POINTER(_VP)]),
    ("olv_graph_create_rmat", _I, [_I, _I, _U64, _I, _U64, ctypes.POINTER(_VP)]),
    ("olv_graph_load", _I, [ctypes.c_char_p, _I, ctypes.POINTER(_VP)]),
    ("olv_graph_destroy", _I, [_VP]),
    ("olv_graph_info", _I, [_VP, ctypes.POINTER(_U32), ctypes.POINTER(_U64), ctypes.POINTER(_I)]),
    ("olv_graph_copy_csr", _I, [_VP, _VP, _VP, _VP]),
    ("olv_graph_set_weights_f32", _I, [_VP, _VP]),
    ("olv_set_stream", _I, [_VP, _VP]),
    ("olv_graph_max_degree_vertex", _I, [_VP, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    ("olv_tune_set", _I, [_VP, ctypes.c_char_p, _D]),
    ("olv_tune_get", _I, [_VP, ctypes.c_char_p, ctypes.POINTER(_D)]),
    ("olv_autotune", _I, [_VP, ctypes.c_char_p, _I]),
    ("olv_autotune_load", _I, [_VP, ctypes.c_char_p, ctypes.POINTER(_I)]),
    ("olv_bfs", _I, [_VP, _U32, _VP, ctypes.POINTER(Stats)]),
    ("olv_bfs_noalloc", _I, [_VP, _VP, _U32, _U64, _U32, _VP, _VP, ctypes.POINTER(Stats)]),
    ("olv_sssp", _I, [_VP, _U32, _VP, ctypes.POINTER(Stats)]),
    ("olv_msbfs", _I, [_VP, _VP, _I, _VP, ctypes.POINTER(Stats)]),
    ("olv_graph_create_er_batch", _I, [_I, _U32, _U32, _U32, _U64, _VP, ctypes.POINTER(_VP)]),
    ("olv_batch_run", _I, [_VP, _VP, _I, _I, _VP, _D, _I, _D, _VP, _VP, _VP,
                           ctypes.POINTER(Stats)]),
    ("olv_pagerank", _I, [_VP, _D, _I, _D, _I, _VP, ctypes.POINTER(Stats)]),
    ("olv_ppr_batch", _I, [_VP, _VP, _I, _D, _I, _D, _VP, ctypes.POINTER(Stats)]),
    ("olv_wpr_forward", _I, [_VP, _VP, _VP, _D, _I, _D, _VP, ctypes.POINTER(_VP),
                             ctypes.POINTER(Stats)]),
    ("olv_wpr_backward", _I, [_VP, _VP, _I, _D, _VP, _VP, ctypes.POINTER(Stats)]),
    ("olv_wpr_ctx_destroy", _I, [_VP]),
    ("olv_write_text", _I, [ctypes.c_char_p, _VP, _U64, _I, _VP, ctypes.POINTER(_U64)]),
    ("olv_graph_save", _I, [_VP, ctypes.c_char_p]),
    ("olv_part_create", _I, [_U32, _U32, _U32, _VP, _VP, _VP, ctypes.POINTER(_VP)]),
    ("olv_part_destroy", _I, [_VP]),
    ("olv_part_set_stream", _I, [_VP, _VP]),
    ("olv_part_bfs_step", _I, [_VP, _VP, _VP, ctypes.c_int32, _VP, ctypes.POINTER(_U64)]),
    ("olv_part_pr_step", _I, [_VP, _VP, _D, _D, _VP, _VP, ctypes.POINTER(_D)]),
]

TEXT_TYPES = {"int32": 0, "uint32": 1, "float32": 2, "float64": 3}


def lib():
    """Load libolive_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m olive_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def symbols():
    return [s[0] for s in _SIGS]


def _check(rc, what):
    if rc != 0:
        msg = lib().olv_last_error().decode(errors="replace")
        raise OliveError(f"{what} failed ({rc}): {msg}")


def _ptr(a):
    """Address of a numpy array or torch tensor (contiguous)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


def _u32(a):
    if hasattr(a, "data_ptr"):
        import torch
        return a.to(torch.int32).contiguous() if a.dtype != torch.int32 else a.contiguous()
    return np.ascontiguousarray(a, dtype=np.uint32)


class Graph:
    """A device-resident graph (olv_graph handle)."""

    def __init__(self, handle):
        self._h = handle
        V, E, wt = _U32(), _U64(), _I()
        _check(lib().olv_graph_info(handle, ctypes.byref(V), ctypes.byref(E), ctypes.byref(wt)),
               "olv_graph_info")
        self.V, self.E, self.weight_type = V.value, E.value, wt.value
        self.last_stats = None

    @classmethod
    def from_csr(cls, rowptr, col, weights=None):
        rowptr, col = _u32(rowptr), _u32(col)
        V = len(rowptr) - 1
        E = len(col)
        wt = W_NONE
        wp = None
        if weights is not None:
            if hasattr(weights, "dtype") and str(weights.dtype) in ("float32", "torch.float32"):
                wt = W_F32
            else:
                wt = W_U32
                weights = _u32(weights)
            wp = _ptr(weights)
        h = _VP()
        _check(lib().olv_graph_create(_ptr(rowptr), _ptr(col) if E else None, wp, wt, V, E,
                                      ctypes.byref(h)), "olv_graph_create")
        return cls(h)

    @classmethod
    def load(cls, path, fmt="edgelist"):
        """Parse an edge-list or DIMACS file on the device."""
        h = _VP()
        _check(lib().olv_graph_load(str(path).encode(), 1 if fmt == "dimacs" else 0,
                                    ctypes.byref(h)), "olv_graph_load")
        return cls(h)

    @classmethod
    def er_batch(cls, count, vmin=1024, vmax=65536, avg_degree=8, seed=1):
        """Block-diagonal batch of ER digraphs; returns (graph, inst_offsets)."""
        off = np.zeros(count + 1, np.uint32)
        h = _VP()
        _check(lib().olv_graph_create_er_batch(count, vmin, vmax, avg_degree, seed, _ptr(off),
                                               ctypes.byref(h)), "olv_graph_create_er_batch")
        return cls(h), off

    @classmethod
    def rmat(cls, scale, edge_factor=16, seed=1, weights=False, wseed=2):
        h = _VP()
        _check(lib().olv_graph_create_rmat(scale, edge_factor, seed, W_U32 if weights else W_NONE,
                                           wseed, ctypes.byref(h)), "olv_graph_create_rmat")
        return cls(h)

    def close(self):
        if getattr(self, "_wctx", None):
            lib().olv_wpr_ctx_destroy(self._wctx)
            self._wctx = None
        if self._h:
            lib().olv_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream):
        """Bind to a CUDA stream (torch.cuda.Stream, raw handle int, or None)."""
        s = getattr(stream, "cuda_stream", stream)
        _check(lib().olv_set_stream(self._h, s), "olv_set_stream")

    def csr(self):
        rowptr = np.empty(self.V + 1, np.uint32)
        col = np.empty(max(self.E, 1), np.uint32)
        w = np.empty(max(self.E, 1), np.float32 if self.weight_type == W_F32 else np.uint32)
        _check(lib().olv_graph_copy_csr(self._h, _ptr(rowptr), _ptr(col),
                                        _ptr(w) if self.weight_type else None),
               "olv_graph_copy_csr")
        return rowptr, col[:self.E], (w[:self.E] if self.weight_type else None)

    def save(self, path):
        """Binary CSR dump (olv_graph_save), read back by Graph.load."""
        _check(lib().olv_graph_save(self._h, str(path).encode()), "olv_graph_save")

    def max_degree_vertex(self):
        v, d = _U32(), _U32()
        _check(lib().olv_graph_max_degree_vertex(self._h, ctypes.byref(v), ctypes.byref(d)),
               "olv_graph_max_degree_vertex")
        return v.value, d.value

    def tune(self, **kw):
        """Set engine tunables (see olv_tune_set); returns the current values."""
        for k, v in kw.items():
            _check(lib().olv_tune_set(self._h, k.encode(), float(v)), f"olv_tune_set({k})")
        out = {}
        for k in ("hub_degree", "piece", "alpha", "beta", "sssp_delta", "sssp_pull", "sssp_relabel",
                  "sssp_sub", "sssp_sub_buckets", "sssp_spt", "sssp_pull_split", "sssp_fuse_end",
                  "sssp_hub_degree", "sssp_piece", "sssp_tail_delta", "sssp_route",
                  "sssp_pull_direct", "ms_alpha", "pr_tile_u", "use_graphs", "levels_per_sync",
                  "batch_cluster"):
            d = _D()
            _check(lib().olv_tune_get(self._h, k.encode(), ctypes.byref(d)), "olv_tune_get")
            out[k] = d.value
        return out

    def autotune(self, json_path=None, reps=3):
        """Time the tunables on this graph, keep the fastest; returns them."""
        _check(lib().olv_autotune(self._h, json_path.encode() if json_path else None, reps),
               "olv_autotune")
        return self.tune()

    def autotune_load(self, json_path):
        """Apply a table written by autotune(); True if it matched this graph."""
        applied = _I()
        _check(lib().olv_autotune_load(self._h, json_path.encode(), ctypes.byref(applied)),
               "olv_autotune_load")
        return bool(applied.value)

    def set_weights_f32(self, w):
        w = np.ascontiguousarray(w, np.float32) if not hasattr(w, "data_ptr") else w.contiguous()
        _check(lib().olv_graph_set_weights_f32(self._h, _ptr(w)), "olv_graph_set_weights_f32")
        self.weight_type = W_F32

    def _out(self, out, dtype):
        return np.empty(self.V, dtype) if out is None else out

    def bfs(self, src, out=None):
        out = self._out(out, np.int32)
        st = Stats()
        _check(lib().olv_bfs(self._h, src, _ptr(out), ctypes.byref(st)), "olv_bfs")
        self.last_stats = st
        return out

    def msbfs(self, srcs, out=None):
        """Levels from up to 64 sources at once: array [len(srcs), V] int32."""
        if not hasattr(srcs, "data_ptr"):
            srcs = np.ascontiguousarray(srcs, np.uint32)
        n = len(srcs)
        if out is None:
            out = np.empty((n, self.V), np.int32)
        st = Stats()
        _check(lib().olv_msbfs(self._h, _ptr(srcs), n, _ptr(out), ctypes.byref(st)), "olv_msbfs")
        self.last_stats = st
        return out

    def batch(self, inst_offsets, seeds=None, K=32, alpha=0.85, max_it=50, tol=1e-7,
              bfs=True, levels_out=None, ppr_out=None):
        """BFS from local vertex 0 and/or K-vector PPR of every instance, in one
        persistent launch.  Returns (levels [V] or None, ppr [V, K] or None,
        iterations per instance)."""
        off = np.ascontiguousarray(inst_offsets, np.uint32)
        count = len(off) - 1
        V = int(off[-1])
        lv = None
        if bfs:
            lv = np.empty(V, np.int32) if levels_out is None else levels_out
        pr = None
        if seeds is not None:
            if not hasattr(seeds, "data_ptr"):
                seeds = np.ascontiguousarray(seeds, np.uint32)
            K = seeds.shape[1]
            pr = np.empty((V, K), np.float32) if ppr_out is None else ppr_out
        iters = np.zeros(count, np.uint32)
        st = Stats()
        _check(lib().olv_batch_run(self._h, _ptr(off), count, K, _ptr(seeds), alpha, max_it, tol,
                                   _ptr(lv), _ptr(pr), _ptr(iters), ctypes.byref(st)),
               "olv_batch_run")
        self.last_stats = st
        return lv, pr, iters

    def sssp(self, src, out=None):
        out = self._out(out, np.uint32)
        st = Stats()
        _check(lib().olv_sssp(self._h, src, _ptr(out), ctypes.byref(st)), "olv_sssp")
        self.last_stats = st
        return out

    def wpr_forward(self, p, w=None, alpha=0.85, max_it=100, tol=0.0, out=None):
        """Weighted PageRank r = (1-alpha) p + alpha P^T r; keeps a context for
        wpr_backward.  w (FP32, CSR order) replaces the graph weights if given."""
        def f32(a):
            if a is None or hasattr(a, "data_ptr"):
                return a
            return np.ascontiguousarray(a, np.float32)
        p, w = f32(p), f32(w)
        out = np.empty(self.V, np.float32) if out is None else out
        if not hasattr(self, "_wctx") or self._wctx is None:
            self._wctx = _VP()
        st = Stats()
        _check(lib().olv_wpr_forward(self._h, _ptr(w), _ptr(p), alpha, max_it, tol, _ptr(out),
                                     ctypes.byref(self._wctx), ctypes.byref(st)),
               "olv_wpr_forward")
        if w is not None:
            self.weight_type = W_F32
        self.last_stats = st
        return out

    def wpr_backward(self, g, max_it=100, tol=0.0, dw_out=None, dp_out=None):
        """dL/dw [E] (CSR order) and dL/dp [V] for L = g . r of the last forward."""
        if not hasattr(g, "data_ptr"):
            g = np.ascontiguousarray(g, np.float32)
        dw = np.empty(self.E, np.float32) if dw_out is None else dw_out
        dp = np.empty(self.V, np.float32) if dp_out is None else dp_out
        st = Stats()
        _check(lib().olv_wpr_backward(self._wctx, _ptr(g), max_it, tol, _ptr(dw), _ptr(dp),
                                      ctypes.byref(st)), "olv_wpr_backward")
        self.last_stats = st
        return dw, dp

    def ppr(self, seeds, alpha=0.85, max_it=50, tol=1e-7, out=None):
        """K <= 32 personalised PageRank vectors (one per seed), advanced
        together: array [V, K] FP32."""
        if not hasattr(seeds, "data_ptr"):
            seeds = np.ascontiguousarray(seeds, np.uint32)
        K = len(seeds)
        out = np.empty((self.V, K), np.float32) if out is None else out
        st = Stats()
        _check(lib().olv_ppr_batch(self._h, _ptr(seeds), K, alpha, max_it, tol, _ptr(out),
                                   ctypes.byref(st)), "olv_ppr_batch")
        self.last_stats = st
        return out

    def pagerank(self, alpha=0.85, max_it=50, tol=1e-7, dangling="uniform", out=None):
        out = self._out(out, np.float32)
        st = Stats()
        _check(lib().olv_pagerank(self._h, alpha, max_it, tol, DANGLING[dangling], _ptr(out),
                                  ctypes.byref(st)), "olv_pagerank")
        self.last_stats = st
        return out
