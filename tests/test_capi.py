"""CPU tests of the C ABI boundary: the library loads and exports every entry
point include/*.h declares; no compute call is made without a GPU."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

import olive_b200 as ob

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(olv_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_loads():
    L = ob.lib()
    assert b"sm_100a" in L.olv_version()


def test_every_declared_symbol_is_exported():
    decl = declared_symbols()
    assert {"olv_bfs", "olv_sssp", "olv_pagerank", "olv_graph_create"} <= decl
    L = ctypes.CDLL(ob.LIB_PATH)
    for name in sorted(decl):
        assert hasattr(L, name), name
    nm = subprocess.run(["nm", "-D", "--defined-only", ob.LIB_PATH], capture_output=True,
                        text=True, check=True).stdout
    exported = set(re.findall(r"\b(olv_[a-z0-9_]+)\b", nm))
    assert decl <= exported
    # every export is declared in a header (no undocumented entry points)
    assert exported <= decl


def test_python_bindings_cover_header():
    assert declared_symbols() == set(ob.symbols())


def test_missing_library_fails_loudly(monkeypatch):
    monkeypatch.setattr(ob, "_lib", None)
    monkeypatch.setattr(ob, "LIB_PATH", "/nonexistent/libolive_b200.so")
    with pytest.raises(ImportError):
        ob.lib()


def test_last_error_is_empty_initially():
    assert ob.lib().olv_last_error() is not None


def test_argument_errors_need_no_gpu():
    L = ob.lib()
    out = ctypes.c_void_p()
    # null rowptr is rejected before any CUDA call
    rc = L.olv_graph_create(None, None, None, 0, 10, 0, ctypes.byref(out))
    assert rc == -1
    assert b"null" in L.olv_last_error()
    rc = L.olv_bfs(None, 0, None, None)
    assert rc == -1
    rc = L.olv_graph_create_rmat(0, 16, 1, 0, 0, ctypes.byref(out))
    assert rc == -1


def test_no_unresolved_library_symbols():
    """Every symbol the library's own translation units reference is defined
    in it (a kernel declared in one .cu file and defined with another
    signature elsewhere would only fail when first called)."""
    nm = subprocess.run(["nm", "-D", "-C", "--undefined-only", ob.LIB_PATH], capture_output=True,
                        text=True, check=True).stdout
    own = [ln for ln in nm.splitlines() if "olv::" in ln or " olv_" in ln]
    assert not own, own
