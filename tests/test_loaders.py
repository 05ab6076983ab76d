"""CPU tests of the source-compatible graph loaders (include/olive/csrGraph.h)
against the reference's loader restated in the oracle and against the
reference's own testCsrGraph (oracle/_ref) where it was built."""
import glob
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "fixture_*.npz")))


@pytest.fixture(scope="module")
def dump_exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "csr_dump")
    cmd = ["g++", "-O1", "-std=c++17", "-w", "-I/usr/local/cuda/include",
           "-I" + os.path.join(ROOT, "include", "olive"),
           os.path.join(ROOT, "tests", "cpp", "csr_dump.cpp"), "-L/usr/local/cuda/lib64",
           "-lcudart_static", "-lpthread", "-ldl", "-lrt", "-o", out]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    return out


def load(exe, path, dimacs=False):
    p = subprocess.run([exe, path] + (["-dimacs"] if dimacs else []), capture_output=True,
                       text=True, check=True)
    lines = p.stdout.split("\n")
    V, E = map(int, lines[0].split())
    rowptr, col = [0], []
    for v in range(V):
        nb = [int(x) for x in lines[1 + v].split()]
        col += nb
        rowptr.append(len(col))
    assert len(col) == E
    return np.array(rowptr, np.uint32), np.array(col, np.uint32)


def _fid(p):
    return os.path.basename(p)[8:-4]


@pytest.mark.parametrize("path", FIXTURES, ids=_fid)
def test_edge_list_loader(dump_exe, tmp_path, path):
    z = np.load(path)
    f = str(tmp_path / "g.txt")
    oracle.write_edge_list(f, z["sorted_rowptr"], z["sorted_col"])
    rp, cl = load(dump_exe, f)
    np.testing.assert_array_equal(rp, z["sorted_rowptr"])
    np.testing.assert_array_equal(cl, z["sorted_col"])


def test_unsorted_edge_list_is_sorted_stably(dump_exe, tmp_path):
    """The reference attaches out-of-order tuples to the wrong row
    (csrGraph.h:149-160); the loader here sorts by source, keeping file order."""
    f = str(tmp_path / "d.txt")
    with open(f, "w") as fh:
        fh.write("# comment\n5 6\n3 1\n0 4\n3 0\n1 2\n0 1\n4 3 17\n")
    rp, cl = load(dump_exe, f)
    np.testing.assert_array_equal(rp, [0, 2, 3, 3, 5, 6])
    np.testing.assert_array_equal(cl, [4, 1, 2, 1, 0, 3])


def _dimacs(tmp_path, V, adj):
    f = str(tmp_path / "g.graph")
    E2 = sum(len(a) for a in adj)
    with open(f, "w") as fh:
        fh.write("# comment\n")
        fh.write(f"{V} {E2 // 2}\n")
        for a in adj:
            fh.write(" ".join(str(x + 1) for x in a) + "\n")
    return f


def test_dimacs_loader(dump_exe, tmp_path):
    """csrGraph.h:177-236: one line per vertex, 1-based ids, E counts undirected
    edges (stored twice)."""
    rp, cl = oracle.grid_csr(6, 7)
    adj = [cl[rp[v]:rp[v + 1]].tolist() for v in range(len(rp) - 1)]
    f = _dimacs(tmp_path, len(adj), adj)
    rp2, cl2 = load(dump_exe, f, dimacs=True)
    np.testing.assert_array_equal(rp2, rp)
    np.testing.assert_array_equal(cl2, cl)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "testCsrGraph")),
                    reason="reference checkers not built (no reference tree at build time)")
def test_dimacs_counts_match_reference_testCsrGraph(tmp_path):
    rp, cl = oracle.grid_csr(5, 5)
    adj = [cl[rp[v]:rp[v + 1]].tolist() for v in range(len(rp) - 1)]
    f = "g.graph"
    path = _dimacs(tmp_path, len(adj), adj)
    ref = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "testCsrGraph"), path, "-dimacs"],
                         capture_output=True, text=True, cwd=str(tmp_path))
    assert f"Nodes:{len(adj)} Edges:{len(cl)}" in ref.stdout
