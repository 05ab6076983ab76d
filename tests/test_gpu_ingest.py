"""Device-side ingest of the reference's text formats (olv_graph_load) against
the reference loader restated in the oracle."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "fixture_*.npz")))


@pytest.fixture(scope="module")
def ob():
    import olive_b200
    return olive_b200


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[8:-4])
def test_edge_list_fixtures(ob, tmp_path, path):
    z = np.load(path)
    f = str(tmp_path / "g.txt")
    w = z["sorted_weights"] if "sorted_weights" in z else None
    oracle.write_edge_list(f, z["sorted_rowptr"], z["sorted_col"], w)
    with ob.Graph.load(f) as g:
        rp, cl, ww = g.csr()
        np.testing.assert_array_equal(rp, z["sorted_rowptr"])
        np.testing.assert_array_equal(cl, z["sorted_col"])
        if w is not None:
            np.testing.assert_array_equal(ww, w)
        for i, s in enumerate(z["bfs_sources"][:4]):
            np.testing.assert_array_equal(g.bfs(int(s)),
                                          oracle.bfs(z["sorted_rowptr"], z["sorted_col"], int(s))[0])


def test_unsorted_comments_and_no_final_newline(ob, tmp_path):
    f = str(tmp_path / "d.txt")
    with open(f, "w") as fh:
        fh.write("# comment\n\n5 6\n3 1\n0 4\n# inner comment\n3 0\n1 2\n  0 1\n4 3")
    rp, cl, _ = oracle.load_edge_list_sorted(f)
    with ob.Graph.load(f) as g:
        grp, gcl, _ = g.csr()
    np.testing.assert_array_equal(grp, rp)
    np.testing.assert_array_equal(gcl, cl)


def test_rmat_file_roundtrip(ob, tmp_path):
    rp, cl = oracle.rmat_csr(14, 16, 3)
    f = str(tmp_path / "r.txt")
    oracle.write_edge_list(f, rp, cl)
    with ob.Graph.load(f) as g:
        grp, gcl, _ = g.csr()
    np.testing.assert_array_equal(grp, rp)
    np.testing.assert_array_equal(gcl, cl)


def test_dimacs(ob, tmp_path):
    rp, cl = oracle.grid_csr(9, 11)
    f = str(tmp_path / "g.graph")
    with open(f, "w") as fh:
        fh.write("% metis comment\n")
        fh.write(f"{len(rp) - 1} {len(cl) // 2}\n")
        for v in range(len(rp) - 1):
            fh.write(" ".join(str(x + 1) for x in cl[rp[v]:rp[v + 1]]) + "\n")
    with ob.Graph.load(f, "dimacs") as g:
        grp, gcl, _ = g.csr()
        np.testing.assert_array_equal(grp, rp)
        np.testing.assert_array_equal(gcl, cl)
        np.testing.assert_array_equal(g.bfs(0), oracle.bfs(rp, cl, 0)[0])


def test_bad_files(ob, tmp_path):
    f = str(tmp_path / "bad.txt")
    with open(f, "w") as fh:
        fh.write("3 2\n0 1\n1 7\n")
    with pytest.raises(ob.OliveError, match="ids >= V"):
        ob.Graph.load(f)
    with pytest.raises(ob.OliveError):
        ob.Graph.load(str(tmp_path / "missing.txt"))
    with open(f, "w") as fh:
        fh.write("# only a comment\n")
    with pytest.raises(ob.OliveError, match="no header"):
        ob.Graph.load(f)
