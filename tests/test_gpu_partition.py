"""The 1-D vertex partition's GPU steps (olv_part_bfs_step / olv_part_pr_step)
through the C ABI: P parts of one graph run on one GPU with the exchange done
in-process (LocalComm), so no kernel waits on another; levels bit-exact
against the oracle BFS, ranks within 1e-6 of the FP64 oracle."""
import numpy as np
import pytest

from olive_b200 import parallel
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ob():
    import torch
    assert torch.cuda.is_available()
    import olive_b200
    return olive_b200


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_partitioned_rmat(ob, parts):
    rp, cl = oracle.rmat_csr(15, 16, 6)
    deg = np.diff(rp.astype(np.int64))
    pg = parallel.PartitionedGraph.build(rp, cl, parts, rank=None, device="cuda")
    try:
        for s in (int(np.argmax(deg)), int(np.flatnonzero(deg > 0)[11])):
            np.testing.assert_array_equal(pg.bfs(s), oracle.bfs(rp, cl, s)[0])
        r, it, res = pg.pagerank(0.85, 30, 1e-9)
        ref, it_ref, res_ref = oracle.pagerank(rp, cl, 0.85, it, 0.0)
        assert np.max(np.abs(r.astype(np.float64) - ref) / ref) < 1e-6
        assert abs(res - res_ref[-1]) <= 1e-3 * res_ref[-1] + 2e-7
        rl, _, _ = pg.pagerank(0.85, 10, 0.0, dangling="leak")
        refl, _ = oracle.pagerank_leak(rp, cl, 10)
        # testPageRank's loop runs iterations 0..9 and counts them the same way
        assert np.max(np.abs(rl.astype(np.float64) - refl) / refl) < 1e-6
    finally:
        pg.close()


def test_partitioned_grid_long_levels_and_odd_sizes(ob):
    rp, cl = oracle.grid_csr(61, 67)          # V not a multiple of 64, 126 levels
    pg = parallel.PartitionedGraph.build(rp, cl, 5, rank=None, device="cuda")
    try:
        for s in (0, 2000, 61 * 67 - 1):
            np.testing.assert_array_equal(pg.bfs(s), oracle.bfs(rp, cl, s)[0])
    finally:
        pg.close()


def test_part_create_rejects_bad_input(ob):
    with pytest.raises(ob.OliveError):
        parallel.GpuPartStep(100, 10, 50, np.zeros(41, np.uint32), np.zeros(0, np.uint32),
                             np.zeros(40, np.uint32))            # lo not a multiple of 64
    with pytest.raises(ob.OliveError):
        parallel.GpuPartStep(100, 0, 2, np.array([0, 1, 2], np.uint32),
                             np.array([5, 100], np.uint32), np.zeros(2, np.uint32))  # id >= V
