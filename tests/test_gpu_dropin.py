"""The reference's own applications (BFS.cu, SSSP.cu, PageRank.cu), compiled
unmodified against include/olive/ (olive_b200/dropin.py), run on the GPU and
compared with the reference checkers' golden outputs, with the header layer's
edge passes forced to push, forced to pull, or chosen by size
(OLIVE_DIRECTION); and the BFS program with the pull opt-ins
(tests/cpp/bfs_pull_optin.cu)."""
import glob
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPS = os.path.join(ROOT, "olive_b200", "_apps")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "fixture_*.npz")))
INF = oracle.INF


def app(name):
    p = os.path.join(APPS, name)
    if not os.path.exists(p):
        pytest.fail(f"{p} missing: build with python -m olive_b200.dropin (needs the "
                    f"reference sources at build time)")
    return p


DIRECTIONS = ["auto", "push", "pull"]


def run(name, args, cwd, direction="auto"):
    env = dict(os.environ, OLIVE_DIRECTION=direction)
    p = subprocess.run([app(name)] + [str(a) for a in args], cwd=cwd, capture_output=True,
                       text=True, timeout=300, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    return p


def _fid(p):
    return os.path.basename(p)[8:-4]


def edge_file(tmp_path, rowptr, col, w=None, name="g.txt"):
    path = os.path.join(str(tmp_path), name)
    oracle.write_edge_list(path, rowptr, col, w)
    return path


@pytest.mark.gpu
@pytest.mark.parametrize("direction", DIRECTIONS)
@pytest.mark.parametrize("path", FIXTURES, ids=_fid)
def test_bfs_app(tmp_path, path, direction):
    z = np.load(path)
    f = edge_file(tmp_path, z["sorted_rowptr"], z["sorted_col"])
    sorted_input = np.array_equal(z["rowptr"], z["sorted_rowptr"])
    for i, s in enumerate(z["bfs_sources"][:4]):
        run("BFS", [f, "-s", s, "-round", 1000000], tmp_path, direction)
        got = np.loadtxt(os.path.join(str(tmp_path), "BFS.txt"), dtype=np.int64, ndmin=1)
        if sorted_input:
            want = z["bfs_levels"][i]
        else:   # the reference mis-builds unsorted input; compare with the sorted CSR
            want, _ = oracle.bfs(z["sorted_rowptr"], z["sorted_col"], int(s))
        np.testing.assert_array_equal(got, want.astype(np.int64))


@pytest.mark.gpu
def test_bfs_app_grid_and_round_limit(tmp_path):
    g = np.load(os.path.join(GOLDEN, "gen_grid_128x128.npz"))
    rp, cl = oracle.grid_csr(128, 128)
    f = edge_file(tmp_path, rp, cl)
    run("BFS", [f, "-s", 0, "-round", 1000000, "-g", 4, "-scan"], tmp_path)
    got = np.loadtxt(os.path.join(str(tmp_path), "BFS.txt"), dtype=np.int64)
    np.testing.assert_array_equal(got, g["bfs_levels"][0].astype(np.int64))
    # BFS.cu's default -round 100 stops after 101 supersteps (BFS.cu:86,142)
    run("BFS", [f, "-s", 0], tmp_path)
    got = np.loadtxt(os.path.join(str(tmp_path), "BFS.txt"), dtype=np.int64)
    want = g["bfs_levels"][0].astype(np.int64)
    want[want > 101] = INF
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("direction", DIRECTIONS)
@pytest.mark.parametrize("path", FIXTURES, ids=_fid)
def test_sssp_app_unit_weights(tmp_path, path, direction):
    """SSSP.cu sets every weight to 1 (SSSP.cu:131): distances are BFS levels."""
    z = np.load(path)
    f = edge_file(tmp_path, z["sorted_rowptr"], z["sorted_col"])
    for s in z["bfs_sources"][:2]:
        run("SSSP", [f, "-s", s, "-round", 1000000], tmp_path, direction)
        got = np.loadtxt(os.path.join(str(tmp_path), "SSSP.txt"), dtype=np.int64, ndmin=1)
        want, _ = oracle.bfs(z["sorted_rowptr"], z["sorted_col"], int(s))
        np.testing.assert_array_equal(got, want.astype(np.int64))


@pytest.mark.gpu
@pytest.mark.parametrize("direction", DIRECTIONS)
@pytest.mark.parametrize("path", FIXTURES, ids=_fid)
def test_pagerank_app(tmp_path, path, direction):
    z = np.load(path)
    if not np.array_equal(z["rowptr"], z["sorted_rowptr"]):
        pytest.skip("testPageRank ran on the mis-built CSR of unsorted input")
    f = edge_file(tmp_path, z["sorted_rowptr"], z["sorted_col"])
    run("PageRank", [f, "-round", 1000], tmp_path, direction)
    got = np.loadtxt(os.path.join(str(tmp_path), "PageRank.txt"), dtype=np.float64, ndmin=1)
    # both sides print "%f"; FP64 atomics may move the last printed digit
    np.testing.assert_allclose(got, z["pr_ranks"], rtol=0, atol=1.01e-6)


def test_csr_app_matches_reference_counts(tmp_path):
    """testCsrGraph built on the header layer reports what the reference's does."""
    for path in FIXTURES[:4]:
        z = np.load(path)
        f = edge_file(tmp_path, z["sorted_rowptr"], z["sorted_col"])
        p = run("testCsrGraph", [f], tmp_path)
        assert f"Nodes:{len(z['rowptr']) - 1} Edges:{len(z['col'])}" in p.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("direction", DIRECTIONS)
def test_apps_on_rmat_every_direction(tmp_path, direction):
    """RMAT-14 (hubs split into pieces in both directions): BFS.cu and SSSP.cu
    levels equal the oracle's, PageRank.cu equals testPageRank's FP64 loop."""
    import olive_b200 as ob
    rp, cl = oracle.rmat_csr(14, 16, 2)
    path = str(tmp_path / "g.bin")
    ob.write_csr_binary(path, rp, cl)
    hub = int(np.argmax(np.diff(rp.astype(np.int64))))
    want, _ = oracle.bfs(rp, cl, hub)
    for name in ("BFS", "SSSP", "BFSPullOptIn"):
        run(name, [path, "-s", hub, "-round", 100000], tmp_path, direction)
        out = "SSSP.txt" if name == "SSSP" else "BFS.txt"
        got = np.loadtxt(os.path.join(str(tmp_path), out), dtype=np.int64)
        np.testing.assert_array_equal(got, want.astype(np.int64), err_msg=name)
    run("PageRank", [path, "-round", 30], tmp_path, direction)
    got = np.loadtxt(os.path.join(str(tmp_path), "PageRank.txt"), dtype=np.float64)
    ref, _ = oracle.pagerank_leak(rp, cl, 31)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1.01e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=_fid)
def test_bfs_pull_optin_app(tmp_path, path):
    """The opt-in pull (unvisited rows only, first parent) gives BFS levels."""
    z = np.load(path)
    f = edge_file(tmp_path, z["sorted_rowptr"], z["sorted_col"])
    for s in z["bfs_sources"][:3]:
        for direction in DIRECTIONS:
            run("BFSPullOptIn", [f, "-s", s, "-round", 1000000], tmp_path, direction)
            got = np.loadtxt(os.path.join(str(tmp_path), "BFS.txt"), dtype=np.int64, ndmin=1)
            want, _ = oracle.bfs(z["sorted_rowptr"], z["sorted_col"], int(s))
            np.testing.assert_array_equal(got, want.astype(np.int64))
