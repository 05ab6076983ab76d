"""Run one workload a few times for a profiler.

    python -m olive_b200.profile_run --workload bfs|sssp|pagerank|msbfs|wpr|batch|ppr --scale 22
    python -m olive_b200.profile_run --workload write-graph --scale 24 --out g.bin

write-graph writes the seeded RMAT graph as a binary CSR file (for the
reference apps built on the header layer, which a profiler then runs
directly) and prints the highest out-degree vertex.

Builds the seeded RMAT graph on the device (scale, edge factor 16, seed 1;
uint32 weights for sssp, lognormal FP32 weights for wpr), then runs the solve
`--runs` times from the highest out-degree vertex (wpr: one forward and one
backward solve of 100 sweeps; batch: 512 ER graphs, BFS plus K=32 PPR, with
--scale ignored).  Supersteps are launched one kernel at a time (the
engine's host-loop mode, `use_graphs=0`) so that a kernel profiler sees each
launch: kernels inside CUDA graphs with conditional nodes are not profiled
node by node.  The kernels are the same as in the graph mode.

The solves run between cudaProfilerStart and cudaProfilerStop, after one
unprofiled solve that builds the per-graph structures (pull lists, row
plans, light/heavy split), so `ncu --profile-from-start off` sees the solve
kernels only (no graph generation, CSC build or sort).
"""
import argparse
import sys

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["bfs", "sssp", "pagerank", "msbfs", "wpr", "batch",
                                           "ppr", "write-graph"], default="bfs")
    ap.add_argument("--out", default="graph.bin", help="write-graph: output path")
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--graphs", action="store_true", help="keep CUDA-graph mode")
    ap.add_argument("--count", type=int, default=512, help="batch: number of ER graphs")
    ap.add_argument("--batch-cluster", type=int, default=1,
                    help="batch: PPR items on thread-block clusters (1) or one CTA each (0)")
    a = ap.parse_args()
    import torch

    import olive_b200 as ob
    if a.workload == "write-graph":
        g = ob.Graph.rmat(a.scale, 16, 1)
        g.save(a.out)
        print(g.max_degree_vertex()[0])
        g.close()
        return
    if a.workload == "batch":
        count, K = a.count, 32
        g, off = ob.Graph.er_batch(count, 1024, 65536, 8, seed=1)
        g.tune(batch_cluster=a.batch_cluster)
        n = np.diff(off.astype(np.int64))
        rng = np.random.default_rng(11)
        seeds = np.stack([rng.integers(0, ni, K) for ni in n]).astype(np.uint32)
        lv = torch.empty(g.V, dtype=torch.int32, device="cuda")
        pr = torch.empty((g.V, K), dtype=torch.float32, device="cuda")
        g.batch(off, seeds, K=K, alpha=0.85, max_it=50, tol=1e-7, levels_out=lv, ppr_out=pr)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        for _ in range(a.runs):
            g.batch(off, seeds, K=K, alpha=0.85, max_it=50, tol=1e-7, levels_out=lv, ppr_out=pr)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(a.workload, g.last_stats.as_dict(), file=sys.stderr)
        g.close()
        return
    g = ob.Graph.rmat(a.scale, 16, 1, weights=a.workload == "sssp", wseed=2)
    if not a.graphs:
        g.tune(use_graphs=0, levels_per_sync=1)
    hub, _ = g.max_degree_vertex()
    out = torch.empty(g.V, dtype=torch.float32 if a.workload in ("pagerank", "wpr") else torch.int32,
                      device="cuda")
    if a.workload == "msbfs":
        rp, _, _ = g.csr()
        deg = np.diff(rp.astype(np.int64))
        srcs = np.random.default_rng(4).choice(np.flatnonzero(deg > 0), 64,
                                               replace=False).astype(np.uint32)
        out = torch.empty((64, g.V), dtype=torch.int32, device="cuda")
    if a.workload == "wpr":
        rng = np.random.default_rng(7)
        w = torch.from_numpy(rng.lognormal(0.0, 1.0, g.E).astype(np.float32)).cuda()
        pn = rng.exponential(1.0, g.V)
        p = torch.from_numpy((pn / pn.sum()).astype(np.float32)).cuda()
        gv = torch.from_numpy(rng.standard_normal(g.V).astype(np.float32)).cuda()
        dw = torch.empty(g.E, dtype=torch.float32, device="cuda")
        dp = torch.empty(g.V, dtype=torch.float32, device="cuda")
        g.wpr_forward(p, w=w, max_it=100, out=out)   # builds the row plans
        g.wpr_backward(gv, max_it=100, dw_out=dw, dp_out=dp)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        for _ in range(a.runs):
            g.wpr_forward(p, w=w, max_it=100, out=out)
            g.wpr_backward(gv, max_it=100, dw_out=dw, dp_out=dp)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(a.workload, g.last_stats.as_dict(), file=sys.stderr)
        g.close()
        return
    if a.workload == "ppr":
        rp, _, _ = g.csr()
        deg = np.diff(rp.astype(np.int64))
        srcs = np.random.default_rng(3).choice(np.flatnonzero(deg > 0), 32,
                                               replace=False).astype(np.uint32)
        out = torch.empty((g.V, 32), dtype=torch.float32, device="cuda")

    def solve():
        if a.workload == "ppr":
            g.ppr(srcs, 0.85, 50, 1e-7, out=out)
        elif a.workload == "bfs":
            g.bfs(hub, out=out)
        elif a.workload == "sssp":
            g.sssp(hub, out=out)
        elif a.workload == "msbfs":
            g.msbfs(srcs, out=out)
        else:
            g.pagerank(0.85, 50, 1e-7, out=out)
    solve()   # first call: builds the per-graph pull and row structures
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(a.runs):
        solve()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(a.workload, g.last_stats.as_dict(), file=sys.stderr)
    g.close()


if __name__ == "__main__":
    main()
