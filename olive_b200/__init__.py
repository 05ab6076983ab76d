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

__all__ = ["Graph", "OliveError", "lib", "INF", "Stats"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libolive_b200.so")
INF = 0x7FFFFFFF

W_NONE, W_U32, W_F32 = 0, 1, 2
DANGLING = {"uniform": 0, "leak": 1}


class OliveError(RuntimeError):
    pass


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
    ("olv_graph_destroy", _I, [_VP]),
    ("olv_graph_info", _I, [_VP, ctypes.POINTER(_U32), ctypes.POINTER(_U64), ctypes.POINTER(_I)]),
    ("olv_graph_copy_csr", _I, [_VP, _VP, _VP, _VP]),
    ("olv_graph_set_weights_f32", _I, [_VP, _VP]),
    ("olv_set_stream", _I, [_VP, _VP]),
    ("olv_graph_max_degree_vertex", _I, [_VP, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    ("olv_tune_set", _I, [_VP, ctypes.c_char_p, _D]),
    ("olv_tune_get", _I, [_VP, ctypes.c_char_p, ctypes.POINTER(_D)]),
    ("olv_bfs", _I, [_VP, _U32, _VP, ctypes.POINTER(Stats)]),
    ("olv_sssp", _I, [_VP, _U32, _VP, ctypes.POINTER(Stats)]),
    ("olv_pagerank", _I, [_VP, _D, _I, _D, _I, _VP, ctypes.POINTER(Stats)]),
]


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
    def rmat(cls, scale, edge_factor=16, seed=1, weights=False, wseed=2):
        h = _VP()
        _check(lib().olv_graph_create_rmat(scale, edge_factor, seed, W_U32 if weights else W_NONE,
                                           wseed, ctypes.byref(h)), "olv_graph_create_rmat")
        return cls(h)

    def close(self):
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
        for k in ("hub_degree", "piece", "alpha", "beta", "sssp_delta", "use_graphs",
                  "levels_per_sync"):
            d = _D()
            _check(lib().olv_tune_get(self._h, k.encode(), ctypes.byref(d)), "olv_tune_get")
            out[k] = d.value
        return out

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

    def sssp(self, src, out=None):
        out = self._out(out, np.uint32)
        st = Stats()
        _check(lib().olv_sssp(self._h, src, _ptr(out), ctypes.byref(st)), "olv_sssp")
        self.last_stats = st
        return out

    def pagerank(self, alpha=0.85, max_it=50, tol=1e-7, dangling="uniform", out=None):
        out = self._out(out, np.float32)
        st = Stats()
        _check(lib().olv_pagerank(self._h, alpha, max_it, tol, DANGLING[dangling], _ptr(out),
                                  ctypes.byref(st)), "olv_pagerank")
        self.last_stats = st
        return out
