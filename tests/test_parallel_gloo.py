"""The multi-replica host logic on CPU: two gloo ranks share 64 BFS sources
of one graph (disjoint shards, no data-path collective), compute them with the
oracle, and agree on the job's work count and slowest time."""
import os
import socket

import numpy as np
import pytest

from olive_b200 import parallel
from oracle import oracle


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, srcs, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    parallel.init("gloo", timeout_s=60)
    rp, cl = oracle.rmat_csr(10, 16, 7)
    mine = parallel.shard(srcs, rank, world)
    edges = sum(oracle.bfs(rp, cl, int(s))[1] for s in mine)
    total = parallel.sum_over_ranks(edges)
    slowest = parallel.max_over_ranks(1.0 + rank)
    q.put((rank, [int(s) for s in mine], edges, total, slowest))
    parallel.finish()


def test_shard_partitions():
    items = list(range(64))
    for world in (1, 2, 3, 8):
        parts = [parallel.shard(items, r, world) for r in range(world)]
        assert sum(parts, []) == items
        assert max(map(len, parts)) - min(map(len, parts)) <= 1


def test_two_gloo_ranks_replica_sharding():
    import torch.multiprocessing as mp
    rp, cl = oracle.rmat_csr(10, 16, 7)
    deg = np.diff(rp.astype(np.int64))
    srcs = np.random.default_rng(4).choice(np.flatnonzero(deg > 0), 64, replace=False).tolist()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, srcs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = sum(oracle.bfs(rp, cl, int(s))[1] for s in srcs)
    assert out[0][1] + out[1][1] == srcs                      # disjoint, complete shards
    assert out[0][2] + out[1][2] == want
    assert out[0][3] == out[1][3] == want                     # both ranks agree on the total
    assert out[0][4] == out[1][4] == 2.0                      # slowest rank's time


# ------------------------------------------------- 1-D vertex partition --
INF = 0x7FFFFFFF


class NumpyPartStep:
    """The local work of one part in numpy (the CPU stand-in for the GPU's
    olv_part_* kernels in these host-logic tests)."""

    def __init__(self, V, lo, hi, colptr, rowidx, outdeg):
        self.lo, self.hi = lo, hi
        self.cp = np.asarray(colptr, np.int64)
        self.ri = np.asarray(rowidx, np.int64)
        self.od = np.asarray(outdeg, np.int64)

    def bfs(self, frontier, level, next_level, next_words):
        f = frontier.numpy().view(np.uint64)
        lv = level.numpy()
        nw = next_words.numpy().view(np.uint64)
        nw[:] = 0
        found = 0
        for v in range(self.hi - self.lo):
            if lv[v] != INF:
                continue
            u = self.ri[self.cp[v]:self.cp[v + 1]]
            if len(u) and np.any((f[u >> 6] >> (u & 63).astype(np.uint64)) & np.uint64(1)):
                lv[v] = next_level
                nw[v >> 6] |= np.uint64(1) << np.uint64(v & 63)
                found += 1
        return found

    def pagerank(self, contrib, base, alpha, rank, contrib_out):
        c = contrib.numpy().astype(np.float64)
        rk = rank.numpy()
        s = np.array([c[self.ri[self.cp[v]:self.cp[v + 1]]].sum()
                      for v in range(self.hi - self.lo)])
        nr = (base + alpha * s).astype(np.float32)
        res = float(np.abs(nr.astype(np.float64) - rk).sum())
        rk[:] = nr
        out = contrib_out.numpy()
        out[:] = np.where(self.od > 0, nr / np.maximum(self.od, 1), 0).astype(np.float32)
        return res, float(nr[self.od == 0].astype(np.float64).sum())


def test_partition_ranges_balanced_and_aligned():
    rp, cl = oracle.rmat_csr(12, 16, 3)
    colptr, rowidx = parallel.reverse_csr(rp, cl)
    V = len(rp) - 1
    for world in (1, 2, 3, 8):
        rg = parallel.partition_ranges(colptr, world)
        assert rg[0][0] == 0 and rg[-1][1] == V
        assert all(a[1] == b[0] for a, b in zip(rg, rg[1:]))
        assert all(lo % 64 == 0 for lo, _ in rg)
        ins = [int(colptr[hi]) - int(colptr[lo]) for lo, hi in rg]
        assert max(ins) - min(ins) <= len(cl) // world // 2 + 4096


def test_partitioned_bfs_and_pagerank_in_one_process():
    rp, cl = oracle.rmat_csr(11, 16, 5)
    hub = int(np.argmax(np.diff(rp.astype(np.int64))))
    for parts in (1, 3):
        pg = parallel.PartitionedGraph.build(rp, cl, parts, rank=None, device="cpu",
                                             step_factory=NumpyPartStep)
        np.testing.assert_array_equal(pg.bfs(hub), oracle.bfs(rp, cl, hub)[0])
        r, it, _ = pg.pagerank(0.85, 20, 0.0)
        ref, _, _ = oracle.pagerank(rp, cl, 0.85, it, 0.0)
        assert it == 20 and np.max(np.abs(r - ref) / ref) < 1e-5


def _part_worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    parallel.init("gloo", timeout_s=60)
    rp, cl = oracle.rmat_csr(11, 16, 5)
    hub = int(np.argmax(np.diff(rp.astype(np.int64))))
    pg = parallel.PartitionedGraph.build(rp, cl, world, rank=rank, device="cpu",
                                         step_factory=NumpyPartStep)
    lv = pg.bfs(hub)
    pr, it, res = pg.pagerank(0.85, 30, 1e-6)
    q.put((rank, lv, pr, it, res, pg.ranges))
    parallel.finish()


def test_two_gloo_ranks_partitioned_bfs_and_pagerank():
    """Each rank holds half the vertices; levels and ranks gathered on every
    rank equal the oracle's."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_part_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rp, cl = oracle.rmat_csr(11, 16, 5)
    hub = int(np.argmax(np.diff(rp.astype(np.int64))))
    ref, _ = oracle.bfs(rp, cl, hub)
    (_, lv0, pr0, it0, res0, rg), (_, lv1, pr1, it1, res1, _) = out
    assert rg[0][1] == rg[1][0] and rg[0][1] % 64 == 0
    np.testing.assert_array_equal(lv0, ref)
    np.testing.assert_array_equal(lv1, ref)
    assert it0 == it1 and res0 == res1 and np.array_equal(pr0, pr1)
    pref, _, _ = oracle.pagerank(rp, cl, 0.85, it0, 0.0)
    assert np.max(np.abs(pr0 - pref) / pref) < 1e-5
