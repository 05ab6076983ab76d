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
