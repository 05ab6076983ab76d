"""Parity at the sizes the benchmark times, through the C ABI:

* SSSP and BFS on RMAT-24 ef16 (uint32 weights U[1,255], wseed 2) from the
  highest out-degree vertex: bit-exact against serial Dijkstra and the
  restated testBFS queue BFS, plus the shortest-path certificate;
* 64-source BFS on the same graph (sources as the benchmark draws them): four
  rows against the oracle BFS, all 64 against solo GPU BFS runs;
* PageRank on RMAT-22: FP32 within 1e-6 max relative error of the FP64 oracle
  after the same number of iterations;
* the 512-instance Erdos-Renyi batch: every instance's BFS bit-exact, every
  PPR-32 vector within FP32 tolerance of the FP64 oracle after the same
  iterations;
* weighted PageRank forward on RMAT-20 against the FP64 oracle;
* a graph of more than 16,776,960 vertices (the size past which the
  reference's 65,535-block launch cap, utils.h:68, skips vertices): C ABI
  BFS/SSSP/PageRank and the reference's BFS.cu and SSSP.cu apps compiled
  unmodified against the header layer.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
INF = oracle.INF
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPS = os.path.join(ROOT, "olive_b200", "_apps")


@pytest.fixture(scope="module")
def ob():
    import torch
    assert torch.cuda.is_available()
    import olive_b200
    return olive_b200


@pytest.fixture(scope="module")
def rmat24(ob):
    g = ob.Graph.rmat(24, 16, 1, weights=True, wseed=2)
    rp, cl, w = g.csr()
    hub, _ = g.max_degree_vertex()
    yield g, rp, cl, w, hub
    g.close()


def test_sssp_rmat24_vs_dijkstra(rmat24):
    g, rp, cl, w, hub = rmat24
    assert g.V == 1 << 24 and g.E > 250_000_000
    np.testing.assert_array_equal(w[:1000], oracle.uint_weights(1000, 2))
    d = g.sssp(hub)
    st = g.last_stats
    ref, e_ref, _, nset = oracle.dijkstra(rp, cl, w, hub)
    np.testing.assert_array_equal(d, ref)
    assert st.edges_traversed == e_ref and st.vertices_reached == nset
    assert oracle.sp_certificate(rp, cl, d, hub, w) is None
    # own-id run (no renumbering) and the push-only heavy step agree
    g.tune(sssp_relabel=0)
    try:
        np.testing.assert_array_equal(g.sssp(hub), ref)
    finally:
        g.tune(sssp_relabel=1)
    g.tune(sssp_pull=0)
    try:
        np.testing.assert_array_equal(g.sssp(hub), ref)
    finally:
        g.tune(sssp_pull=1)


def test_bfs_rmat24_vs_oracle_and_certificate(rmat24):
    g, rp, cl, _, hub = rmat24
    deg = np.diff(rp.astype(np.int64))
    other = int(np.flatnonzero(deg == 1)[0])   # a low-degree source
    for s in (hub, other):
        lv = g.bfs(s)
        ref, e_ref = oracle.bfs(rp, cl, s)
        np.testing.assert_array_equal(lv, ref)
        assert g.last_stats.edges_traversed == e_ref
        assert oracle.sp_certificate(rp, cl, lv, s) is None


def test_msbfs64_rmat24(ob, rmat24):
    import torch
    g, rp, cl, _, _ = rmat24
    deg = np.diff(rp.astype(np.int64))
    srcs = np.random.default_rng(4).choice(np.flatnonzero(deg > 0), 64,
                                           replace=False).astype(np.uint32)
    out = torch.empty((64, g.V), dtype=torch.int32, device="cuda")
    g.msbfs(torch.from_numpy(srcs.astype(np.int32)).cuda(), out=out)
    e_ms = g.last_stats.edges_traversed
    solo = torch.empty(g.V, dtype=torch.int32, device="cuda")
    e_solo = 0
    for s in range(64):
        g.bfs(int(srcs[s]), out=solo)
        e_solo += g.last_stats.edges_traversed
        assert torch.equal(out[s], solo), f"row {s} differs from the solo run"
    assert e_ms == e_solo
    for s in (0, 1, 31, 63):
        ref, _ = oracle.bfs(rp, cl, int(srcs[s]))
        np.testing.assert_array_equal(out[s].cpu().numpy(), ref, err_msg=f"row {s}")


def test_pagerank_rmat22_vs_fp64(ob):
    with ob.Graph.rmat(22, 16, 1) as g:
        rp, cl, _ = g.csr()
        r = g.pagerank(0.85, 50, 1e-7)
        it = g.last_stats.iterations
        ref, it_ref, res = oracle.pagerank(rp, cl, 0.85, it, 0.0)
        assert it_ref == it
        rel = np.abs(r.astype(np.float64) - ref) / ref
        assert rel.max() < 1e-6, rel.max()
        assert abs(g.last_stats.residual - res[-1]) <= 1e-3 * res[-1] + 2e-7


def test_batch_er512_every_instance(ob):
    count, K = 512, 32
    g, off = ob.Graph.er_batch(count, 1024, 65536, 8, seed=1)
    try:
        rp, cl, _ = g.csr()
        n = np.diff(off.astype(np.int64))
        np.testing.assert_array_equal(n, oracle.er_batch_sizes(count, 1024, 65536, 1))
        rng = np.random.default_rng(11)   # the benchmark's seeds
        seeds = np.stack([rng.integers(0, ni, K) for ni in n]).astype(np.uint32)
        lv, pr, iters = g.batch(off, seeds, K=K, alpha=0.85, max_it=50, tol=1e-7)
    finally:
        g.close()
    for i in range(count):
        b, e = int(off[i]), int(off[i + 1])
        lrp = (rp[b:e + 1] - rp[b]).astype(np.uint32)
        lcl = (cl[rp[b]:rp[e]] - b).astype(np.uint32)
        ref, _ = oracle.bfs(lrp, lcl, 0)
        np.testing.assert_array_equal(lv[b:e], ref, err_msg=f"instance {i}")
    # the oracle runs each instance for the iterations the GPU ran
    pref, pit = oracle.ppr_batch(rp, cl, off, seeds, 0.85, iters.astype(np.int32), 0.0)
    np.testing.assert_array_equal(pit, iters)
    assert iters.max() <= 50 and iters.min() >= 2
    for i in range(count):
        b, e = int(off[i]), int(off[i + 1])
        np.testing.assert_allclose(pr[b:e].astype(np.float64), pref[b:e], rtol=2e-5, atol=2e-7,
                                   err_msg=f"instance {i}")


def test_wpr_forward_rmat20_vs_oracle(ob):
    with ob.Graph.rmat(20, 16, 1) as g:
        rp, cl, _ = g.csr()
        rng = np.random.default_rng(7)    # the benchmark's inputs
        w = rng.lognormal(0.0, 1.0, g.E).astype(np.float32)
        pn = rng.exponential(1.0, g.V)
        p = (pn / pn.sum()).astype(np.float32)
        r = g.wpr_forward(p, w=w, alpha=0.85, max_it=100)
    ref = oracle.wpr_forward(rp, cl, w.astype(np.float64), p.astype(np.float64), 0.85, 100)
    rel = np.abs(r.astype(np.float64) - ref) / ref
    assert rel.max() < 1e-5, rel.max()


# ------------------------------------------------- past 16,776,960 vertices --
BIG_V = (1 << 24) + 4099     # not a multiple of 32 or 256


def _tree_csr(V):
    """Binary-heap tree with child edges v -> 2v+1, 2v+2 and a back edge to
    the parent: BFS level of v from 0 is floor(log2(v + 1))."""
    v = np.arange(V, dtype=np.int64)
    kids = np.stack([2 * v + 1, 2 * v + 2], 1)
    par = np.where(v > 0, (v - 1) // 2, -1)[:, None]
    nb = np.concatenate([par, kids], 1)       # parent first, then children
    ok = (nb >= 0) & (nb < V)
    rp = np.zeros(V + 1, np.uint32)
    rp[1:] = np.cumsum(ok.sum(1))
    return rp, nb[ok].astype(np.uint32)


@pytest.fixture(scope="module")
def big_tree():
    rp, cl = _tree_csr(BIG_V)
    return rp, cl


def _tree_levels(V):
    return np.floor(np.log2(np.arange(V, dtype=np.float64) + 1)).astype(np.int32)


def test_past_2pow24_vertices_c_abi(ob, big_tree):
    rp, cl = big_tree
    w = oracle.uint_weights(len(cl), 17)
    with ob.Graph.from_csr(rp, cl, w) as g:
        assert g.V == BIG_V
        lv = g.bfs(0)
        np.testing.assert_array_equal(lv, _tree_levels(BIG_V))
        last = BIG_V - 1
        lv2 = g.bfs(last)
        assert lv2[0] == _tree_levels(BIG_V)[last]
        assert oracle.sp_certificate(rp, cl, lv2, last) is None
        d = g.sssp(last)
        assert (d != INF).all()
        assert oracle.sp_certificate(rp, cl, d, last, w) is None
        r = g.pagerank(0.85, 10, 0.0)
        ref, _, _ = oracle.pagerank(rp, cl, 0.85, 10, 0.0)
        rel = np.abs(r.astype(np.float64) - ref) / ref
        assert rel.max() < 1e-6, rel.max()


def _app(name):
    p = os.path.join(APPS, name)
    if not os.path.exists(p):
        pytest.fail(f"{p} missing: build with python -m olive_b200.dropin (needs the "
                    f"reference sources at build time)")
    return p


def _read_ints(path):
    import pandas as pd
    return pd.read_csv(path, header=None, dtype=np.int64)[0].values


@pytest.mark.parametrize("name", ["BFS", "SSSP"])
def test_past_2pow24_vertices_header_layer(ob, big_tree, tmp_path, name):
    """The reference apps, compiled unmodified against include/olive/, reach
    every vertex of the tree (the reference's own kernels never processed the
    last vertices at this size)."""
    rp, cl = big_tree
    path = str(tmp_path / "tree.bin")
    ob.write_csr_binary(path, rp, cl)
    p = subprocess.run([_app(name), path, "-s", "0", "-round", "1000"], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    got = _read_ints(str(tmp_path / f"{name}.txt"))
    np.testing.assert_array_equal(got, _tree_levels(BIG_V).astype(np.int64))


def test_ppr32_rmat22_vs_oracle(ob):
    """32 personalised PageRank vectors on RMAT-22 (the benchmarked size)."""
    with ob.Graph.rmat(22, 16, 1) as g:
        rp, cl, _ = g.csr()
        deg = np.diff(rp.astype(np.int64))
        seeds = np.random.default_rng(3).choice(np.flatnonzero(deg > 0), 32,
                                                replace=False).astype(np.uint32)
        out = g.ppr(seeds, 0.85, 50, 1e-7)
        it = g.last_stats.iterations
    # the oracle in four parallel slices of 8 vectors (FP64, same iterations)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(4) as ex:
        parts = list(ex.map(lambda k: oracle.ppr(rp, cl, seeds[k:k + 8], 0.85, it, 0.0),
                            range(0, 32, 8)))
    ref = np.concatenate([p[0] for p in parts], axis=1)
    got = out.astype(np.float64)
    for k in range(32):
        r, gk = ref[:, k], got[:, k]
        assert np.max(np.abs(gk - r)) <= 1e-6 * np.max(np.abs(r)), k
        nz = r > 0
        assert np.all(gk[~nz] == 0)
        assert np.max(np.abs(gk[nz] - r[nz]) / r[nz]) < 1e-5, k
