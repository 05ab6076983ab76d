"""Block-diagonal batches run by one persistent kernel: every instance equals
its solo run (bitwise) and the CPU oracle (BFS bit-exact, PPR within FP32
tolerance of the FP64 oracle)."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
INF = oracle.INF


@pytest.fixture(scope="module")
def ob():
    import torch
    assert torch.cuda.is_available()
    import olive_b200
    return olive_b200


def instance_csr(rp, cl, off, i):
    b, e = int(off[i]), int(off[i + 1])
    lrp = (rp[b:e + 1] - rp[b]).astype(np.uint32)
    lcl = (cl[rp[b]:rp[e]] - b).astype(np.uint32)
    return lrp, lcl


def draw_seeds(off, K, seed=0):
    rng = np.random.default_rng(seed)
    n = np.diff(off.astype(np.int64))
    return np.stack([rng.integers(0, ni, K) for ni in n]).astype(np.uint32)


@pytest.fixture(scope="module")
def small_batch(ob):
    g, off = ob.Graph.er_batch(24, 300, 3000, 8, seed=3)
    rp, cl, _ = g.csr()
    yield g, off, rp, cl
    g.close()


def test_er_generator_properties(small_batch):
    g, off, rp, cl = small_batch
    n = np.diff(off.astype(np.int64))
    assert n.min() >= 300 and n.max() <= 3000
    for i in range(len(n)):
        lrp, lcl = instance_csr(rp, cl, off, i)
        assert len(lcl) == 8 * n[i]
        src = np.repeat(np.arange(n[i]), np.diff(lrp.astype(np.int64)))
        assert not np.any(src == lcl)                      # no self-loops
        keys = src * n[i] + lcl
        assert len(np.unique(keys)) == len(keys)           # no duplicates
        assert lcl.max() < n[i]                            # block diagonal


def test_er_generator_equals_oracle_restatement(small_batch):
    """The library's batch generator and the oracle's restatement (which the
    reference arm of bench.py uses) draw the same instances."""
    g, off, rp, cl = small_batch
    n = np.diff(off.astype(np.int64))
    np.testing.assert_array_equal(n, oracle.er_batch_sizes(24, 300, 3000, 3))
    for i in range(len(n)):
        lrp, lcl = instance_csr(rp, cl, off, i)
        orp, ocl = oracle.er_batch_instance(i, int(n[i]), 8, 3)
        np.testing.assert_array_equal(lrp, orp)
        np.testing.assert_array_equal(lcl, ocl)


def test_batch_bfs_and_ppr_vs_oracle(ob, small_batch):
    g, off, rp, cl = small_batch
    K = 32
    seeds = draw_seeds(off, K)
    lv, pr, iters = g.batch(off, seeds, alpha=0.85, max_it=30, tol=0.0)
    assert np.all(iters == 30)
    for i in range(len(off) - 1):
        lrp, lcl = instance_csr(rp, cl, off, i)
        ref, _ = oracle.bfs(lrp, lcl, 0)
        np.testing.assert_array_equal(lv[off[i]:off[i + 1]], ref, err_msg=f"instance {i}")
        pref, it = oracle.ppr(lrp, lcl, seeds[i], 0.85, 30, 0.0)
        assert it == 30
        got = pr[off[i]:off[i + 1]].astype(np.float64)
        np.testing.assert_allclose(got, pref, rtol=2e-5, atol=2e-7)


def test_batch_instances_equal_solo_runs(ob, small_batch):
    g, off, rp, cl = small_batch
    K = 32
    seeds = draw_seeds(off, K, 1)
    lv, pr, iters = g.batch(off, seeds, max_it=50, tol=1e-7)
    for i in (0, 5, 11, 23):
        lrp, lcl = instance_csr(rp, cl, off, i)
        with ob.Graph.from_csr(lrp, lcl) as solo:
            slv, spr, sit = solo.batch(np.array([0, len(lrp) - 1], np.uint32), seeds[i:i + 1])
        assert sit[0] == iters[i]
        assert slv.tobytes() == lv[off[i]:off[i + 1]].tobytes()
        assert spr.tobytes() == pr[off[i]:off[i + 1]].tobytes()
    # and a second batch run is identical
    lv2, pr2, it2 = g.batch(off, seeds, max_it=50, tol=1e-7)
    assert lv2.tobytes() == lv.tobytes() and pr2.tobytes() == pr.tobytes()
    assert np.array_equal(it2, iters)


def test_batch_bfs_only_and_ppr_only(ob, small_batch):
    g, off, rp, cl = small_batch
    lv, pr, _ = g.batch(off, None)
    assert pr is None
    lv2, pr2, _ = g.batch(off, draw_seeds(off, 8), bfs=False, max_it=10, tol=0.0)
    assert lv2 is None and pr2.shape == (off[-1], 8)
    lrp, lcl = instance_csr(rp, cl, off, 2)
    np.testing.assert_array_equal(lv[off[2]:off[3]], oracle.bfs(lrp, lcl, 0)[0])


def test_batch_limits(ob):
    rp, cl = oracle.grid_csr(300, 300)   # one instance of 90,000 vertices: over the limit
    with ob.Graph.from_csr(rp, cl) as g:
        with pytest.raises(ob.OliveError):
            g.batch(np.array([0, 90000], np.uint32), None)
        with pytest.raises(ob.OliveError):
            g.batch(np.array([0, 40000, 90000], np.uint32), np.zeros((2, 33), np.uint32))


def test_batch_rejects_non_block_diagonal(ob):
    rp, cl = oracle.grid_csr(20, 20)
    with ob.Graph.from_csr(rp, cl) as g:
        with pytest.raises(ob.OliveError, match="block-diagonal"):
            g.batch(np.array([0, 200, 400], np.uint32), np.zeros((2, 4), np.uint32), max_it=3)


@pytest.mark.parametrize("cluster", [0, 1, 8])
def test_batch_cluster_and_cta_paths_vs_oracle(ob, small_batch, cluster):
    """Both ways of running the PPR items (one thread-block cluster per item,
    or one CTA per item) agree with the FP64 oracle; each is deterministic."""
    g, off, rp, cl = small_batch
    K = 32
    seeds = draw_seeds(off, K, 5)
    g.tune(batch_cluster=cluster)
    try:
        lv, pr, iters = g.batch(off, seeds, alpha=0.85, max_it=20, tol=0.0)
        lv2, pr2, _ = g.batch(off, seeds, alpha=0.85, max_it=20, tol=0.0)
    finally:
        g.tune(batch_cluster=1)
    assert pr.tobytes() == pr2.tobytes() and lv.tobytes() == lv2.tobytes()
    for i in (0, 7, 23):
        lrp, lcl = instance_csr(rp, cl, off, i)
        np.testing.assert_array_equal(lv[off[i]:off[i + 1]], oracle.bfs(lrp, lcl, 0)[0])
        pref, _ = oracle.ppr(lrp, lcl, seeds[i], 0.85, 20, 0.0)
        np.testing.assert_allclose(pr[off[i]:off[i + 1]].astype(np.float64), pref,
                                   rtol=2e-5, atol=2e-7)
