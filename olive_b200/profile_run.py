"""Run one workload a few times for a profiler.

    python -m olive_b200.profile_run --workload bfs|sssp|pagerank|msbfs --scale 22

Builds the seeded RMAT graph on the device (scale, edge factor 16, seed 1;
uint32 weights for sssp), then runs the solve `--runs` times from the highest
out-degree vertex.  Supersteps are launched one kernel at a time (the
engine's host-loop mode, `use_graphs=0`) so that a kernel profiler sees each
launch: kernels inside CUDA graphs with conditional nodes are not profiled
node by node.  The kernels are the same as in the graph mode.
"""
import argparse
import sys

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["bfs", "sssp", "pagerank", "msbfs"], default="bfs")
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--graphs", action="store_true", help="keep CUDA-graph mode")
    a = ap.parse_args()
    import torch

    import olive_b200 as ob
    g = ob.Graph.rmat(a.scale, 16, 1, weights=a.workload == "sssp", wseed=2)
    if not a.graphs:
        g.tune(use_graphs=0, levels_per_sync=1)
    hub, _ = g.max_degree_vertex()
    out = torch.empty(g.V, dtype=torch.float32 if a.workload == "pagerank" else torch.int32,
                      device="cuda")
    if a.workload == "msbfs":
        rp, _, _ = g.csr()
        deg = np.diff(rp.astype(np.int64))
        srcs = np.random.default_rng(4).choice(np.flatnonzero(deg > 0), 64,
                                               replace=False).astype(np.uint32)
        out = torch.empty((64, g.V), dtype=torch.int32, device="cuda")
    for _ in range(a.runs):
        if a.workload == "bfs":
            g.bfs(hub, out=out)
        elif a.workload == "sssp":
            g.sssp(hub, out=out)
        elif a.workload == "msbfs":
            g.msbfs(srcs, out=out)
        else:
            g.pagerank(0.85, 50, 1e-7, out=out)
    torch.cuda.synchronize()
    print(a.workload, g.last_stats.as_dict(), file=sys.stderr)
    g.close()


if __name__ == "__main__":
    main()
