"""CPU tests: the oracle against the reference's own outputs (golden fixtures
made by tests/golden/make_golden.py from the reference's serial checkers)."""
import glob
import hashlib
import os

import numpy as np
import pytest

from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "fixture_*.npz")))


def _digest(rowptr, col):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rowptr, np.uint32).tobytes())
    h.update(np.ascontiguousarray(col, np.uint32).tobytes())
    return h.hexdigest()


def test_fixtures_present():
    names = {os.path.basename(f) for f in FIXTURES}
    assert len(names) == 9, names


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[8:-4])
def test_bfs_matches_reference_checker(path):
    z = np.load(path)
    for i, s in enumerate(z["bfs_sources"]):
        lv, _ = oracle.bfs(z["rowptr"], z["col"], int(s))
        np.testing.assert_array_equal(lv, z["bfs_levels"][i])


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[8:-4])
def test_pagerank_leak_matches_reference_checker(path):
    z = np.load(path)
    for key, max_it in (("pr", 1000), ("pr50", 50)):
        r, it = oracle.pagerank_leak(z["rowptr"], z["col"], max_it)
        assert it == int(z[f"{key}_iterations"])
        # the reference prints "%f": 6 decimals
        np.testing.assert_allclose(r, z[f"{key}_ranks"], rtol=0, atol=5.0000001e-7)


@pytest.mark.parametrize("name", ["grid_128x128", "rmat10_ef16_s1", "rmat12_ef16_s1"])
def test_generated_graphs_pinned(name):
    z = np.load(os.path.join(GOLDEN, f"gen_{name}.npz"))
    if name.startswith("grid"):
        rp, cl = oracle.grid_csr(128, 128)
    else:
        rp, cl = oracle.rmat_csr(int(name[4:6]), 16, 1)
    assert len(rp) - 1 == int(z["V"]) and len(cl) == int(z["E"])
    assert _digest(rp, cl) == str(z["digest"])
    for i, s in enumerate(z["bfs_sources"]):
        np.testing.assert_array_equal(oracle.bfs(rp, cl, int(s))[0], z["bfs_levels"][i])
    r, it = oracle.pagerank_leak(rp, cl, 50)
    assert it == int(z["pr50_iterations"])
    np.testing.assert_allclose(r, z["pr50_ranks"], rtol=0, atol=5.0000001e-7)


def test_grid_shape():
    rp, cl = oracle.grid_csr(128, 128)
    assert len(rp) == 16385 and len(cl) == 65024
    # neighbours of vertex 129 (row 1, col 1) in (up, left, right, down) order
    assert list(cl[rp[129]:rp[130]]) == [1, 128, 130, 257]


def test_disordered_loader_quirk():
    """csrGraph.h:149-160 attaches out-of-order tuples to the current row; the
    sorted loader does not.  The two CSRs differ on disorderedGraph_9."""
    z = np.load(os.path.join(GOLDEN, "fixture_disorderedGraph_9.npz"))
    assert not np.array_equal(z["rowptr"], z["sorted_rowptr"])
    z2 = np.load(os.path.join(GOLDEN, "fixture_orderedGraph_9.npz"))
    np.testing.assert_array_equal(z2["rowptr"], z2["sorted_rowptr"])
    np.testing.assert_array_equal(z2["col"], z2["sorted_col"])


def test_permutation_is_bijection():
    L = oracle.lib()
    for bits in (1, 2, 5, 10, 13):
        ys = {L.orc_permute(x, bits, 12345) for x in range(1 << bits)}
        assert ys == set(range(1 << bits))


def test_dijkstra_unit_weights_equal_bfs():
    rp, cl = oracle.rmat_csr(11, 16, 3)
    w = np.ones(len(cl), np.uint32)
    for s in (0, 5, 77):
        d, *_ = oracle.dijkstra(rp, cl, w, s)
        lv, _ = oracle.bfs(rp, cl, s)
        np.testing.assert_array_equal(d.astype(np.int64), lv.astype(np.int64))


@pytest.mark.parametrize("threads", [1, 4])
def test_frontier_bellman_ford_equals_dijkstra(threads):
    rp, cl = oracle.rmat_csr(12, 16, 5)
    w = oracle.uint_weights(len(cl), 9)
    assert w.min() >= 1 and w.max() <= 255
    deg = np.diff(rp.astype(np.int64))
    src = int(np.argmax(deg))
    d1, *_ = oracle.dijkstra(rp, cl, w, src)
    d2, edges, _, rounds = oracle.sssp_frontier(rp, cl, w, src, threads=threads)
    np.testing.assert_array_equal(d1, d2)
    assert rounds > 1 and edges >= deg[d1 != oracle.INF].sum()


def test_pagerank_dangling_mass_conserved():
    rp, cl = oracle.rmat_csr(10, 8, 2)
    r, it, res = oracle.pagerank(rp, cl, 0.85, 200, 1e-12)
    assert abs(r.sum() - 1.0) < 1e-9
    assert res[-1] < 1e-12 or it == 200


def test_pagerank_leak_equals_uniform_without_dangling():
    rp, cl = oracle.grid_csr(6, 7)
    r1, _, _ = oracle.pagerank(rp, cl, 0.85, 30, 0.0)
    z = np.zeros(1)
    r2, _ = oracle.pagerank_leak(rp, cl, 30)
    # testPageRank stops when err < 1e-7 (not reached in 30 on this graph)
    np.testing.assert_allclose(r1, r2, rtol=1e-13, atol=0)


def test_ppr_fixed_point():
    rp, cl = oracle.rmat_csr(9, 8, 4)
    seeds = np.array([0, 3, 100], np.uint32)
    r, it = oracle.ppr(rp, cl, seeds, 0.85, 400, 1e-13)
    V = len(rp) - 1
    deg = np.diff(rp.astype(np.int64))
    src = np.repeat(np.arange(V), deg)
    for k, s in enumerate(seeds):
        x = r[:, k]
        y = np.zeros(V)
        np.add.at(y, cl.astype(np.int64), x[src] / deg[src])
        dang = x[deg == 0].sum()
        y *= 0.85
        y[s] += 0.15 + 0.85 * dang
        np.testing.assert_allclose(x, y, rtol=1e-9, atol=1e-14)
        assert abs(x.sum() - 1) < 1e-9


def test_wpr_adjoint_matches_dense_solve():
    rng = np.random.default_rng(0)
    rp, cl = oracle.rmat_csr(7, 8, 6)
    V, E = len(rp) - 1, len(cl)
    w = rng.lognormal(0, 1, E)
    p = rng.exponential(1, V)
    p /= p.sum()
    g = rng.standard_normal(V)
    a = 0.85
    deg = np.diff(rp.astype(np.int64))
    src = np.repeat(np.arange(V), deg)
    W = np.zeros(V)
    np.add.at(W, src, w)
    P = np.zeros((V, V))
    np.add.at(P, (src, cl.astype(np.int64)), w / W[src])
    A = np.eye(V) - a * P.T
    r_dense = np.linalg.solve(A, (1 - a) * p)
    r = oracle.wpr_forward(rp, cl, w, p, a, 400)
    np.testing.assert_allclose(r, r_dense, rtol=1e-10, atol=1e-15)
    lam, dw, dp = oracle.wpr_backward(rp, cl, w, r, g, a, 400)
    lam_dense = np.linalg.solve(np.eye(V) - a * P, g)
    np.testing.assert_allclose(lam, lam_dense, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(dp, (1 - a) * lam_dense, rtol=1e-9, atol=1e-12)
    # dL/dw by central finite differences on a few edges
    for e in rng.choice(E, 5, replace=False):
        h = 1e-6 * w[e]
        wp_, wm_ = w.copy(), w.copy()
        wp_[e] += h
        wm_[e] -= h
        fp = g @ oracle.wpr_forward(rp, cl, wp_, p, a, 400)
        fm = g @ oracle.wpr_forward(rp, cl, wm_, p, a, 400)
        fd = (fp - fm) / (2 * h)
        assert abs(fd - dw[e]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9


def test_er_batch_restatement_properties():
    """Oracle restatement of the batch generator: exact edge counts, no
    self-loops or duplicates, rows sorted; a 2-vertex instance saturates."""
    sizes = oracle.er_batch_sizes(5, 40, 700, 1)
    assert sizes.min() >= 40 and sizes.max() <= 700
    for i, n in enumerate(sizes):
        rp, col = oracle.er_batch_instance(i, int(n), 8, 1)
        assert rp[-1] == 8 * n and len(col) == 8 * n
        src = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
        assert not np.any(src == col)
        keys = src * n + col
        assert (np.diff(keys) > 0).all()     # sorted by (u, v), no duplicates
    rp, col = oracle.er_batch_instance(0, 2, 8, 3)
    np.testing.assert_array_equal(rp, [0, 1, 2])
    np.testing.assert_array_equal(col, [1, 0])


# ------------------------------------------- certificate, batched PPR, writer --
def test_sp_certificate_accepts_exact_and_rejects_perturbed():
    rp, cl = oracle.rmat_csr(12, 16, 3)
    lv, _ = oracle.bfs(rp, cl, 0)
    assert oracle.sp_certificate(rp, cl, lv, 0) is None
    reached = np.flatnonzero((lv != oracle.INF) & (lv > 0))
    for delta in (1, -1):
        bad = lv.copy()
        bad[reached[len(reached) // 2]] += delta
        assert oracle.sp_certificate(rp, cl, bad, 0) is not None
    w = oracle.uint_weights(len(cl), 5)
    d, *_ = oracle.dijkstra(rp, cl, w, 0)
    assert oracle.sp_certificate(rp, cl, d, 0, w) is None
    bad = d.copy()
    bad[np.flatnonzero(d == oracle.INF)[0]] = 7        # an unreachable vertex marked reached
    assert oracle.sp_certificate(rp, cl, bad, 0, w)[1] == "no tight in-edge"
    bad = d.copy()
    bad[0] = 1
    assert oracle.sp_certificate(rp, cl, bad, 0, w)[1] == "source not at 0"


def test_ppr_batch_equals_per_instance_runs():
    sizes = oracle.er_batch_sizes(5, 200, 900, 4)
    parts = [oracle.er_batch_instance(i, int(n), 8, 4) for i, n in enumerate(sizes)]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)
    rp = [np.zeros(1, np.int64)]
    base = 0
    for lrp, _ in parts:
        rp.append(lrp[1:].astype(np.int64) + base)
        base += int(lrp[-1])
    rp = np.concatenate(rp).astype(np.uint32)
    cl = np.concatenate([lcl + off[i] for i, (_, lcl) in enumerate(parts)]).astype(np.uint32)
    rng = np.random.default_rng(1)
    seeds = np.stack([rng.integers(0, n, 8) for n in sizes]).astype(np.uint32)
    r, it = oracle.ppr_batch(rp, cl, off, seeds, 0.85, 40, 1e-7)
    for i, (lrp, lcl) in enumerate(parts):
        ri, iti = oracle.ppr(lrp, lcl, seeds[i], 0.85, 40, 1e-7)
        assert iti == it[i]
        assert np.array_equal(ri, r[off[i]:off[i + 1]])
    _, it2 = oracle.ppr_batch(rp, cl, off, seeds, 0.85, np.array([1, 2, 3, 4, 5]), 0.0)
    assert list(it2) == [1, 2, 3, 4, 5]


def test_edge_list_writer_round_trips_through_the_reference_loader(tmp_path):
    rp, cl = oracle.rmat_csr(9, 8, 2)
    path = str(tmp_path / "g.txt")
    oracle.write_edge_list(path, rp, cl)
    rp2, cl2 = oracle.load_edge_list_ref(path)[:2]
    assert np.array_equal(rp2, rp) and np.array_equal(cl2, cl)
