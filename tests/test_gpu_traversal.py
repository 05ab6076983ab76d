"""GPU parity tests: BFS, SSSP and PageRank through the C ABI against the
reference checkers' golden outputs and the CPU oracle."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "fixture_*.npz")))
INF = oracle.INF


@pytest.fixture(scope="module")
def ob():
    import torch
    assert torch.cuda.is_available()
    import olive_b200
    return olive_b200


def _fid(p):
    return os.path.basename(p)[8:-4]


# ------------------------------------------------------------------ BFS --
@pytest.mark.parametrize("path", FIXTURES, ids=_fid)
def test_bfs_reference_fixtures_every_source(ob, path):
    """Bit-exact against testBFS on the CSR the reference loader builds."""
    z = np.load(path)
    with ob.Graph.from_csr(z["rowptr"], z["col"]) as g:
        for i, s in enumerate(z["bfs_sources"]):
            lv = g.bfs(int(s))
            np.testing.assert_array_equal(lv, z["bfs_levels"][i], err_msg=f"source {s}")


def test_bfs_grid_128(ob):
    z = np.load(os.path.join(GOLDEN, "gen_grid_128x128.npz"))
    rp, cl = oracle.grid_csr(128, 128)
    with ob.Graph.from_csr(rp, cl) as g:
        for i, s in enumerate(z["bfs_sources"]):
            np.testing.assert_array_equal(g.bfs(int(s)), z["bfs_levels"][i])
        g.bfs(0)
        # 254 levels beyond the source (the reference app stops at -round 100)
        assert g.last_stats.iterations == int(z["bfs_levels"][0].max()) + 1
        assert g.last_stats.vertices_reached == 16384
        assert g.last_stats.edges_traversed == 65024


@pytest.mark.parametrize("scale", [10, 12])
def test_bfs_rmat_golden_and_generator(ob, scale):
    z = np.load(os.path.join(GOLDEN, f"gen_rmat{scale}_ef16_s1.npz"))
    rp, cl = oracle.rmat_csr(scale, 16, 1)
    with ob.Graph.rmat(scale, 16, 1) as g:
        grp, gcl, _ = g.csr()
        np.testing.assert_array_equal(grp, rp)   # device generator == CPU restatement
        np.testing.assert_array_equal(gcl, cl)
        for i, s in enumerate(z["bfs_sources"]):
            np.testing.assert_array_equal(g.bfs(int(s)), z["bfs_levels"][i])


@pytest.mark.parametrize("scale,seed", [(14, 1), (16, 7)])
def test_bfs_rmat_vs_oracle(ob, scale, seed):
    with ob.Graph.rmat(scale, 16, seed) as g:
        rp, cl, _ = g.csr()
        hub, _ = g.max_degree_vertex()
        deg = np.diff(rp.astype(np.int64))
        rng = np.random.default_rng(scale)
        for s in [hub] + rng.choice(np.flatnonzero(deg > 0), 4, replace=False).tolist():
            ref, e_ref = oracle.bfs(rp, cl, int(s))
            np.testing.assert_array_equal(g.bfs(int(s)), ref)
            st = g.last_stats
            assert st.edges_traversed == e_ref
            assert st.vertices_reached == int((ref != INF).sum())


def test_bfs_device_output_and_repeat(ob):
    import torch
    with ob.Graph.rmat(15, 16, 3) as g:
        rp, cl, _ = g.csr()
        hub, _ = g.max_degree_vertex()
        ref, _ = oracle.bfs(rp, cl, hub)
        out = torch.empty(g.V, dtype=torch.int32, device="cuda")
        for _ in range(3):
            g.bfs(hub, out=out)
            np.testing.assert_array_equal(out.cpu().numpy(), ref)
        # unaligned device output (offset by one element)
        big = torch.empty(g.V + 1, dtype=torch.int32, device="cuda")
        g.bfs(hub, out=big[1:])
        np.testing.assert_array_equal(big[1:].cpu().numpy(), ref)


def test_bfs_source_out_of_range(ob):
    rp, cl = oracle.grid_csr(4, 4)
    with ob.Graph.from_csr(rp, cl) as g:
        with pytest.raises(ob.OliveError):
            g.bfs(16)


def test_bfs_unsorted_rows_and_duplicates(ob):
    """Rows in any order, duplicate edges and self-loops give the same levels."""
    rng = np.random.default_rng(5)
    V = 3000
    src = rng.integers(0, V, 40000)
    dst = rng.integers(0, V, 40000)
    dst[:500] = src[:500]                      # self-loops
    src = np.concatenate([src, src[:1000]])    # duplicates
    dst = np.concatenate([dst, dst[:1000]])
    order = np.argsort(src, kind="stable")
    rp = np.zeros(V + 1, np.int64)
    np.add.at(rp, src + 1, 1)
    rp = np.cumsum(rp).astype(np.uint32)
    cl = dst[order].astype(np.uint32)
    with ob.Graph.from_csr(rp, cl) as g:
        for s in (0, 17, 2999):
            np.testing.assert_array_equal(g.bfs(s), oracle.bfs(rp, cl, s)[0])


# ----------------------------------------------------------------- SSSP --
@pytest.mark.parametrize("path", [p for p in FIXTURES if "weights" in np.load(p)], ids=_fid)
def test_sssp_weighted_fixtures(ob, path):
    z = np.load(path)
    rp, cl, w = z["sorted_rowptr"], z["sorted_col"], z["sorted_weights"]
    with ob.Graph.from_csr(rp, cl, w) as g:
        for s in range(0, len(rp) - 1, 7):
            ref, *_ = oracle.dijkstra(rp, cl, w, s)
            np.testing.assert_array_equal(g.sssp(s), ref)


@pytest.mark.parametrize("path", FIXTURES, ids=_fid)
def test_sssp_unit_weights_equal_reference_bfs(ob, path):
    """SSSP.cu forces every weight to 1 (SSSP.cu:131): distances are BFS levels."""
    z = np.load(path)
    w = np.ones(len(z["col"]), np.uint32)
    with ob.Graph.from_csr(z["rowptr"], z["col"], w) as g:
        for i, s in enumerate(z["bfs_sources"][:20]):
            d = g.sssp(int(s))
            np.testing.assert_array_equal(d.astype(np.int64),
                                          z["bfs_levels"][i].astype(np.int64))


@pytest.mark.parametrize("pull", [0, 1])
@pytest.mark.parametrize("scale,seed", [(12, 1), (16, 2), (18, 3)])
def test_sssp_rmat_vs_dijkstra(ob, scale, seed, pull):
    """Heavy edges by push only (pull=0) or by the in-edge pull where it reads
    fewer edges (pull=1, the default): the same distances either way."""
    with ob.Graph.rmat(scale, 16, seed, weights=True, wseed=seed + 10) as g:
        g.tune(sssp_pull=pull)
        rp, cl, w = g.csr()
        np.testing.assert_array_equal(w, oracle.uint_weights(len(cl), seed + 10))
        hub, _ = g.max_degree_vertex()
        deg = np.diff(rp.astype(np.int64))
        for s in (hub, int(np.flatnonzero(deg > 0)[3])):
            ref, e_ref, _, nset = oracle.dijkstra(rp, cl, w, s)
            np.testing.assert_array_equal(g.sssp(s), ref)
            st = g.last_stats
            assert st.edges_traversed == e_ref and st.vertices_reached == nset
            if not pull:   # push relaxes every out-edge of a reached vertex at least once
                assert st.edges_relaxed >= st.edges_traversed
        if pull and scale >= 16:
            # the pull reads far fewer edges than the push from the hub
            g.sssp(hub)
            relaxed_pull = g.last_stats.edges_relaxed
            g.tune(sssp_pull=0)
            g.sssp(hub)
            assert relaxed_pull < g.last_stats.edges_relaxed


@pytest.mark.parametrize("hub,piece", [(32, 32), (4096, 4096)])
def test_sssp_hub_pieces_vs_dijkstra(ob, hub, piece):
    """Rows over sssp_hub_degree go to warp pieces of sssp_piece edges: every
    split gives the same distances (32/32 puts most RMAT rows in pieces)."""
    with ob.Graph.rmat(16, 16, 4, weights=True, wseed=9) as g:
        g.tune(sssp_hub_degree=hub, sssp_piece=piece)
        rp, cl, w = g.csr()
        hubv, _ = g.max_degree_vertex()
        for s in (hubv, 5):
            np.testing.assert_array_equal(g.sssp(s), oracle.dijkstra(rp, cl, w, s)[0])


@pytest.mark.parametrize("spt,fuse", [(1, 0), (1, 1), (2, 1), (4, 0), (4, 1), (8, 1)])
def test_sssp_chunk_shape_and_fused_end_vs_dijkstra(ob, spt, fuse):
    """Relax chunks of 256 x spt queued sources, and the superstep's end step
    run by the pieces kernel's last CTA (fuse 1) or by its own launch: the
    same distances, inside the CUDA graph and in the host loop."""
    with ob.Graph.rmat(16, 16, 5, weights=True, wseed=4) as g:
        g.tune(sssp_spt=spt, sssp_fuse_end=fuse, sssp_hub_degree=64, sssp_piece=64)
        rp, cl, w = g.csr()
        hub, _ = g.max_degree_vertex()
        deg = np.diff(rp.astype(np.int64))
        for s in (hub, int(np.flatnonzero(deg > 0)[3])):
            ref = oracle.dijkstra(rp, cl, w, s)[0]
            np.testing.assert_array_equal(g.sssp(s), ref)
        g.tune(use_graphs=0)
        np.testing.assert_array_equal(g.sssp(hub), oracle.dijkstra(rp, cl, w, hub)[0])
        g.tune(use_graphs=1, sssp_sub=8)
        np.testing.assert_array_equal(g.sssp(hub), oracle.dijkstra(rp, cl, w, hub)[0])


@pytest.mark.parametrize("tail", [0, 65, 256, 1000, 1 << 30])
def test_sssp_wide_tail_buckets_vs_dijkstra(ob, tail):
    """Buckets after the first of width sssp_tail_delta relaxing every edge
    (0 and widths <= delta: light/heavy throughout; 2^30: one Bellman-Ford
    bucket after the first): Dijkstra's distances from the hub and from a
    low-degree source, with the pull or push heavy step, sub-buckets in the
    first bucket, in the graph and in the host loop."""
    with ob.Graph.rmat(16, 16, 6, weights=True, wseed=8) as g:
        g.tune(sssp_tail_delta=tail)
        rp, cl, w = g.csr()
        hub, _ = g.max_degree_vertex()
        deg = np.diff(rp.astype(np.int64))
        ref_hub = oracle.dijkstra(rp, cl, w, hub)[0]
        for s in (hub, int(np.flatnonzero(deg == 1)[0])):
            np.testing.assert_array_equal(g.sssp(s), oracle.dijkstra(rp, cl, w, s)[0])
        for kw in ({"sssp_pull": 0}, {"sssp_sub": 16}, {"use_graphs": 0}, {"sssp_relabel": 0},
                   {"sssp_route": 0}, {"sssp_pull_split": 0}, {"sssp_pull_direct": 0}):
            base = g.tune()
            g.tune(**kw)
            np.testing.assert_array_equal(g.sssp(hub), ref_hub, err_msg=str(kw))
            g.tune(**{k: base[k] for k in kw})


@pytest.mark.parametrize("path", [p for p in FIXTURES if "weights" in np.load(p)], ids=_fid)
def test_sssp_wide_tail_on_fixtures(ob, path):
    """The weighted fixtures with narrow and wide buckets after the first."""
    z = np.load(path)
    rp, cl, w = z["sorted_rowptr"], z["sorted_col"], z["sorted_weights"]
    with ob.Graph.from_csr(rp, cl, w) as g:
        for tail in (2, 300):
            g.tune(sssp_delta=1, sssp_tail_delta=tail)
            for s in range(0, len(rp) - 1, 5):
                ref, *_ = oracle.dijkstra(rp, cl, w, s)
                np.testing.assert_array_equal(g.sssp(s), ref, err_msg=f"tail {tail} source {s}")


def test_sssp_chunk_shape_rejects_bad_values(ob):
    with ob.Graph.rmat(8, 4, 1, weights=True) as g:
        for bad in (0, 3, 16):
            with pytest.raises(ob.OliveError):
                g.tune(sssp_spt=bad)


@pytest.mark.parametrize("sub,nsub", [(0, 1), (4, 1), (8, 2), (16, 1), (1, 3), (500, 1)])
def test_sssp_sub_buckets_vs_dijkstra(ob, sub, nsub):
    """The first heavy buckets' light phase in sub-buckets of every width
    (0 and widths >= delta: none) gives Dijkstra's distances, with the pull
    heavy step or the push."""
    with ob.Graph.rmat(15, 16, 8, weights=True, wseed=12) as g:
        g.tune(sssp_sub=sub, sssp_sub_buckets=nsub)
        rp, cl, w = g.csr()
        hub, _ = g.max_degree_vertex()
        for s in (hub, int(np.flatnonzero(np.diff(rp.astype(np.int64)) > 0)[9])):
            ref = oracle.dijkstra(rp, cl, w, s)[0]
            np.testing.assert_array_equal(g.sssp(s), ref)
        g.tune(sssp_pull=0)
        np.testing.assert_array_equal(g.sssp(hub), oracle.dijkstra(rp, cl, w, hub)[0])


def test_sssp_relabel_on_off_same_handle(ob):
    """Renumbered (default) and own-id runs on one handle, toggled back and
    forth, into host, device and unaligned device outputs."""
    import torch
    with ob.Graph.rmat(16, 16, 6, weights=True, wseed=3) as g:
        rp, cl, w = g.csr()
        hub, _ = g.max_degree_vertex()
        ref = oracle.dijkstra(rp, cl, w, hub)[0]
        for relabel in (1, 0, 1):
            g.tune(sssp_relabel=relabel)
            np.testing.assert_array_equal(g.sssp(hub), ref)
            big = torch.empty(g.V + 1, dtype=torch.int32, device="cuda")
            g.sssp(hub, out=big[1:])
            np.testing.assert_array_equal(big[1:].cpu().numpy().astype(np.uint32), ref)
        np.testing.assert_array_equal(g.sssp(7), oracle.dijkstra(rp, cl, w, 7)[0])


def _core_graph(n_core=300, n_tail=40, seed=5):
    """Source -> core by light edges, a complete core of heavy edges (most of
    E, all landing on settled vertices), core -> four targets with 300 heavy
    in-edges each (warp-read in-rows) and -> tail vertices with 3 in-edges
    each (thread-read in-rows); targets and tail lead on into later buckets,
    and two unreachable vertices point at a target."""
    rng = np.random.default_rng(seed)
    src = 0
    core = np.arange(1, n_core + 1)
    tgt = np.arange(n_core + 1, n_core + 5)
    tail = np.arange(n_core + 5, n_core + 5 + n_tail)
    far = np.arange(tail[-1] + 1, tail[-1] + 1 + 50)
    unr = np.array([far[-1] + 1, far[-1] + 2])
    V = int(unr[-1]) + 1
    e = []
    e += [(src, int(c), int(rng.integers(1, 20))) for c in core]
    e += [(int(a), int(b), int(rng.integers(100, 400))) for a in core for b in core if a != b]
    e += [(int(a), int(t), int(rng.integers(65, 900))) for t in tgt for a in core]
    e += [(int(a), int(t), int(rng.integers(65, 900))) for t in tail
          for a in rng.choice(core, 3, replace=False)]
    e += [(int(t), int(f), int(rng.integers(1, 300))) for t in np.concatenate([tgt, tail])
          for f in rng.choice(far, 4, replace=False)]
    e += [(int(f), int(rng.choice(far)), int(rng.integers(1, 100))) for f in far]
    e += [(int(u), int(tgt[0]), 1) for u in unr]
    e.sort()
    a = np.array(e, dtype=np.int64)
    rp = np.zeros(V + 1, np.uint32)
    np.add.at(rp, a[:, 0] + 1, 1)
    return np.cumsum(rp).astype(np.uint32), a[:, 1].astype(np.uint32), a[:, 2].astype(np.uint32)


@pytest.mark.parametrize("pull", [0, 1])
def test_sssp_pull_superstep_long_and_short_in_rows(ob, pull):
    rp, cl, w = _core_graph()
    ref, e_ref, _, nset = oracle.dijkstra(rp, cl, w, 0)
    with ob.Graph.from_csr(rp, cl, w) as g:
        g.tune(sssp_pull=pull)
        np.testing.assert_array_equal(g.sssp(0), ref)
        st = g.last_stats
        assert st.edges_traversed == e_ref and st.vertices_reached == nset
        if pull:   # the core's heavy edges were not relaxed one by one
            assert st.edges_relaxed < (len(cl) * 3) // 4
        for s in (1, 7):
            np.testing.assert_array_equal(g.sssp(s), oracle.dijkstra(rp, cl, w, s)[0])


def test_sssp_needs_weights(ob):
    rp, cl = oracle.grid_csr(3, 3)
    with ob.Graph.from_csr(rp, cl) as g:
        with pytest.raises(ob.OliveError):
            g.sssp(0)


# ------------------------------------------------------------- PageRank --
@pytest.mark.parametrize("path", FIXTURES, ids=_fid)
def test_pagerank_leak_matches_reference_checker(ob, path):
    """dangling='leak' reproduces testPageRank (printed with %f)."""
    z = np.load(path)
    # testPageRank converged on every fixture: it ran pr_iterations + 1 sweeps
    # (it breaks before counting the last one, testPageRank.cu:102-103)
    sweeps = int(z["pr_iterations"]) + 1
    with ob.Graph.from_csr(z["rowptr"], z["col"]) as g:
        r = g.pagerank(0.85, sweeps, 0.0, dangling="leak")
        assert g.last_stats.iterations == sweeps
        np.testing.assert_allclose(r, z["pr_ranks"], rtol=0, atol=6e-7)
        r50 = g.pagerank(0.85, 50, 0.0, dangling="leak")
        if int(z["pr50_iterations"]) == 50:
            np.testing.assert_allclose(r50, z["pr50_ranks"], rtol=0, atol=6e-7)


@pytest.mark.parametrize("scale,seed", [(12, 1), (16, 3), (18, 4)])
def test_pagerank_fp32_vs_fp64_oracle(ob, scale, seed):
    """FP32 ranks within 1e-6 max relative error of the FP64 oracle after the
    same number of iterations (dangling mass redistributed)."""
    with ob.Graph.rmat(scale, 16, seed) as g:
        rp, cl, _ = g.csr()
        r = g.pagerank(0.85, 50, 1e-7)
        it = g.last_stats.iterations
        ref, it_ref, res = oracle.pagerank(rp, cl, 0.85, it, 0.0)
        assert it_ref == it
        rel = np.abs(r.astype(np.float64) - ref) / ref
        assert rel.max() < 1e-6, rel.max()
        # the GPU residual is summed from FP32 ranks: ~1e-7 absolute noise
        assert abs(g.last_stats.residual - res[-1]) <= 1e-3 * res[-1] + 2e-7


@pytest.mark.parametrize("tile_u", [1, 4, 16, 32])
def test_pagerank_and_wpr_every_row_grouping(ob, tile_u):
    """Every row grouping of the tile plans keeps PageRank within 1e-6 of the
    FP64 oracle and weighted PageRank within 1e-5."""
    with ob.Graph.rmat(15, 16, 11) as g:
        g.tune(pr_tile_u=tile_u)
        rp, cl, _ = g.csr()
        r = g.pagerank(0.85, 25, 0.0)
        ref, _, _ = oracle.pagerank(rp, cl, 0.85, 25, 0.0)
        assert np.max(np.abs(r - ref) / ref) < 1e-6
        rng = np.random.default_rng(tile_u)
        w = rng.lognormal(0, 1, g.E).astype(np.float32)
        p = np.full(g.V, 1.0 / g.V, np.float32)
        rw = g.wpr_forward(p, w=w, max_it=60)
        rref = oracle.wpr_forward(rp, cl, w.astype(np.float64), p.astype(np.float64), 0.85, 60)
        assert np.max(np.abs(rw - rref) / rref) < 1e-5
        g.tune(pr_tile_u=8)   # plans dropped: the backward asks for a new forward
        with pytest.raises(ob.OliveError, match="run the forward again"):
            g.wpr_backward(np.ones(g.V, np.float32), max_it=5)


def test_pagerank_deterministic(ob):
    with ob.Graph.rmat(17, 16, 9) as g:
        a = g.pagerank(0.85, 30, 0.0)
        b = g.pagerank(0.85, 30, 0.0)
        assert a.tobytes() == b.tobytes()


def test_pagerank_tolerance_stop(ob):
    rp, cl = oracle.grid_csr(20, 20)
    with ob.Graph.from_csr(rp, cl) as g:
        g.pagerank(0.85, 1000, 1e-5)
        it = g.last_stats.iterations
        _, it_ref, res = oracle.pagerank(rp, cl, 0.85, 1000, 1e-5)
        assert abs(it - it_ref) <= 1
        assert g.last_stats.residual < 1e-5


# ------------------------------------------------------------------ msBFS --
@pytest.mark.parametrize("scale,seed,n", [(12, 1, 64), (16, 5, 64), (14, 2, 5), (10, 3, 1)])
def test_msbfs_rows_equal_solo_bfs(ob, scale, seed, n):
    with ob.Graph.rmat(scale, 16, seed) as g:
        rp, cl, _ = g.csr()
        deg = np.diff(rp.astype(np.int64))
        rng = np.random.default_rng(seed)
        srcs = rng.choice(np.flatnonzero(deg > 0), n, replace=False).astype(np.uint32)
        lv = g.msbfs(srcs)
        st = g.last_stats
        e_tot = 0
        for s in range(n):
            ref, e = oracle.bfs(rp, cl, int(srcs[s]))
            np.testing.assert_array_equal(lv[s], ref, err_msg=f"row {s}")
            e_tot += e
            np.testing.assert_array_equal(lv[s], g.bfs(int(srcs[s])))
        assert st.edges_traversed == e_tot


def test_msbfs_fixtures_duplicates_and_device_output(ob):
    import torch
    for path in FIXTURES:
        z = np.load(path)
        srcs = z["bfs_sources"][:64].astype(np.uint32)
        with ob.Graph.from_csr(z["rowptr"], z["col"]) as g:
            lv = g.msbfs(srcs)
            np.testing.assert_array_equal(lv, z["bfs_levels"][:64])
            dup = np.array([srcs[0], srcs[0], srcs[-1]], np.uint32)
            out = torch.empty((3, g.V), dtype=torch.int32, device="cuda")
            g.msbfs(dup, out=out)
            o = out.cpu().numpy()
            np.testing.assert_array_equal(o[0], z["bfs_levels"][0])
            np.testing.assert_array_equal(o[1], z["bfs_levels"][0])


@pytest.mark.parametrize("rows,cols,n", [(37, 29, 64), (11, 3, 40), (128, 128, 33)])
def test_msbfs_long_diameter_grids(ob, rows, cols, n):
    """Grids: levels far past the 16 stored level slots, V not a multiple of 32."""
    rp, cl = oracle.grid_csr(rows, cols)
    V = rows * cols
    srcs = np.random.default_rng(rows).choice(V, min(n, V), replace=False).astype(np.uint32)
    with ob.Graph.from_csr(rp, cl) as g:
        lv = g.msbfs(srcs)
        for s in range(len(srcs)):
            ref, _ = oracle.bfs(rp, cl, int(srcs[s]))
            np.testing.assert_array_equal(lv[s], ref, err_msg=f"row {s}")


def test_msbfs_bad_arguments(ob):
    rp, cl = oracle.grid_csr(4, 4)
    with ob.Graph.from_csr(rp, cl) as g:
        with pytest.raises(ob.OliveError):
            g.msbfs(np.arange(65, dtype=np.uint32) % 16)
        with pytest.raises(ob.OliveError):
            g.msbfs(np.array([16], np.uint32))


# -------------------------------------------------------------- autotune --
def test_autotune_keeps_results_and_roundtrips(ob, tmp_path):
    with ob.Graph.rmat(14, 16, 3, weights=True, wseed=4) as g:
        rp, cl, w = g.csr()
        hub, _ = g.max_degree_vertex()
        path = str(tmp_path / "tune.json")
        best = g.autotune(path, reps=1)
        assert best["hub_degree"] in (256, 1024, 4096)
        assert best["sssp_hub_degree"] in (128, 256, 1024) and best["sssp_piece"] in (256, 1024)
        assert best["pr_tile_u"] in (4, 8, 16) and best["ms_alpha"] in (5, 10, 20, 40)
        assert best["sssp_sub"] in (0, 8, 16) and best["sssp_tail_delta"] in (0, 256, 1024, 4096)
        assert best["sssp_delta"] in (8, 16, 24, 32, 64, 128, 256)
        np.testing.assert_array_equal(g.bfs(hub), oracle.bfs(rp, cl, hub)[0])
        np.testing.assert_array_equal(g.sssp(hub), oracle.dijkstra(rp, cl, w, hub)[0])
        txt = open(path).read()
        assert '"key"' in txt and "sssp_delta" in txt and "pr_tile_u" in txt and "ms_alpha" in txt
        r = g.pagerank(0.85, 30, 0.0)
        ref, _, _ = oracle.pagerank(rp, cl, 0.85, 30, 0.0)
        assert np.max(np.abs(r - ref) / ref) < 1e-6
    with ob.Graph.rmat(14, 16, 3, weights=True, wseed=4) as g2:
        g2.tune(hub_degree=4096, sssp_delta=16, sssp_hub_degree=4096, sssp_piece=4096,
                sssp_tail_delta=7, pr_tile_u=32, ms_alpha=7)
        assert g2.autotune_load(path)
        assert g2.tune() == best
    with ob.Graph.rmat(13, 16, 3) as g3:       # another graph: table not applied
        before = g3.tune()
        assert not g3.autotune_load(path)
        assert g3.tune() == before
