#!/usr/bin/env python
"""Benchmark of the olive_b200 frontier engine on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sssp|bfs|pagerank] [--scale S]

Default workload: single-source shortest paths (frontier Bellman-Ford with
atomicMin, SSSP.cu semantics) on an RMAT graph of scale 24, edge factor 16,
(a,b,c,d) = (.57,.19,.19,.05), uint32 weights uniform in [1,255], from the
highest out-degree vertex.  A step is one complete solve on the resident
graph.  The metric is GTEPS = (sum of out-degrees of reached vertices) / time.
BFS on the same graph is measured in the same run and reported under "bfs".

One process per GPU (torchrun); every rank runs its own replica of the
workload (the traversal does not shard: "replicas only"), `value` sums the
ranks' edges over the slowest rank's time.  Rank 0 prints one JSON line.

--impl reference times the reference's algorithm on the host cores: the
CPU restatement of SSSP.cu's frontier Bellman-Ford (all host threads), of
testBFS.cu's queue BFS, or of testPageRank.cu's FP64 PageRank, on the same
synthetic graph built on the host.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

INF = 0x7FFFFFFF
PEAK_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["sssp", "bfs", "pagerank"], default="sssp")
    ap.add_argument("--scale", type=int, default=None)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="bound of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    a = ap.parse_args()
    if a.scale is None:
        a.scale = 22 if a.workload == "pagerank" else 24
    a.warmup = max(a.warmup, 3) if a.impl == "ours" else a.warmup
    return a


def metric_name(w, scale):
    if w == "sssp":
        return f"SSSP GTEPS, RMAT-{scale} ef16, uint32 weights U[1,255], src = max out-degree"
    if w == "bfs":
        return f"BFS GTEPS, RMAT-{scale} ef16, src = max out-degree"
    return f"PageRank GE/s/iter, RMAT-{scale} ef16, alpha 0.85, FP32, dangling redistributed"


def workload_config(a, V=None, E=None, src=None, extra=None):
    c = {"workload": f"{a.workload}-rmat{a.scale}", "scale": a.scale, "edge_factor": 16,
         "rmat_abcd": [0.57, 0.19, 0.19, 0.05], "seed": a.seed, "V": V, "E": E,
         "parallelism": f"replicas x{a.gpus} (one whole graph per GPU)"}
    if a.workload == "sssp":
        c.update(weights="uint32 U[1,255], wseed 2", source=src)
    elif a.workload == "bfs":
        c.update(source=src)
    else:
        c.update(alpha=0.85, max_it=50, tol=1e-7, dangling="uniform")
    c["l2"] = "inputs larger than L2 (CSR/CSC arrays >= 1 GB per pass), no flush needed"
    if extra:
        c.update(extra)
    return c


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return PEAK_FALLBACK_GBS, "fallback 6.65 TB/s"


class ClockSampler:
    """nvidia-smi clock/throttle samples taken while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(prefix="olv_clocks_", suffix=".csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        self.t0 = time.time()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sms, mx, reasons, pw = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
                pw.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sms)) if sms else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sms),
                "power_w_max": max(pw) if pw else None}


# ----------------------------------------------------------------- ours --
def run_ours(a, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    import olive_b200 as ob

    stream = torch.cuda.current_stream()
    weights = a.workload == "sssp"
    g = ob.Graph.rmat(a.scale, 16, a.seed, weights=weights, wseed=2)
    g.set_stream(stream)
    src, _ = g.max_degree_vertex()
    V, E = g.V, g.E
    out = torch.empty(V, dtype=torch.float32 if a.workload == "pagerank" else torch.int32,
                      device="cuda")

    def step(dst):
        if a.workload == "sssp":
            return g.sssp(src, out=dst)
        if a.workload == "bfs":
            return g.bfs(src, out=dst)
        return g.pagerank(0.85, 50, 1e-7, out=dst)

    for _ in range(a.warmup):
        step(out)
    torch.cuda.synchronize()
    st = g.last_stats
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)   # let the sampler start before the timed region
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dev_ms = []
    for _ in range(a.steps):
        step(out)
        dev_ms.append(g.last_stats.device_ms)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1) / a.steps
    clk = clocks.stop()
    st = g.last_stats
    t_ms = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(t_ms, op=dist.ReduceOp.MAX)
    ms_max = float(t_ms.item())

    if a.workload == "pagerank":
        units = E * st.iterations                    # edge visits per solve
        value = world * units / (ms_max * 1e-3) / 1e9  # GE/s/iter aggregate
        unit = "GE/s/iter"
        alg_bytes = (8 * E + 20 * V) * st.iterations
        bytes_formula = "(8 B/edge + 20 B/vertex) per iteration"
    else:
        units = st.edges_traversed
        value = world * units / (ms_max * 1e-3) / 1e9
        unit = "GTEPS"
        per_edge = 12 if a.workload == "sssp" else 8
        alg_bytes = per_edge * st.edges_traversed + 20 * st.vertices_reached
        bytes_formula = f"{per_edge} B/traversed edge + 20 B/reached vertex"
    peak, peak_src = peaks()
    kern_ms = float(np.median(dev_ms))
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None,
                "kernel": f"whole {a.workload} solve (all kernels of one call, CUDA graph)",
                "algorithmic_bytes": int(alg_bytes), "bytes_formula": bytes_formula,
                "peak_source": peak_src, "kernel_ms": round(kern_ms, 4)}

    # launches of our kernels per step (kernel nodes executed by the graph)
    if a.workload == "sssp":
        per_step = 2 + 5 * st.iterations + 1
    elif a.workload == "bfs":
        per_step = 2 + 6 * st.iterations
    else:
        per_step = 2 + 2 * st.iterations
    launches = per_step * a.steps

    # end to end through the public API: host (pinned) output buffer, D2H inside
    host_out = torch.empty(V, dtype=out.dtype, pin_memory=True)
    step(host_out)
    x0 = torch.cuda.Event(enable_timing=True)
    x1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    x0.record(stream)
    t_wall = time.perf_counter()
    for _ in range(a.steps):
        step(host_out)
    x1.record(stream)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t_wall) * 1e3 / a.steps
    e2e_ms = max(x0.elapsed_time(x1) / a.steps, wall_ms)
    t_e = torch.tensor([e2e_ms], device="cuda")
    if world > 1:
        dist.all_reduce(t_e, op=dist.ReduceOp.MAX)
    e2e_ms = float(t_e.item())
    e2e = {"value": round(world * units / (e2e_ms * 1e-3) / 1e9, 3), "unit": unit,
           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(V * 4),
           "ms_per_step": round(e2e_ms, 4),
           "note": "olv_* call with a pinned host output buffer; the per-call input is the "
                   "source id passed by value; graph resident as after Oliver::readGraph"}

    extra = {}
    # BFS on the same graph, reported beside the SSSP headline
    if a.workload == "sssp":
        lv = torch.empty(V, dtype=torch.int32, device="cuda")
        for _ in range(3):
            g.bfs(src, out=lv)
        bm = []
        for _ in range(max(a.steps, 5)):
            g.bfs(src, out=lv)
            bm.append(g.last_stats.device_ms)
        bs = g.last_stats
        bms = float(np.median(bm))
        bbytes = 8 * bs.edges_traversed + 20 * bs.vertices_reached
        extra["bfs"] = {"metric": metric_name("bfs", a.scale), "value": round(
            bs.edges_traversed / (bms * 1e-3) / 1e9, 2), "unit": "GTEPS", "ms": round(bms, 4),
            "levels": bs.iterations, "pull_levels": bs.pull_steps,
            "roofline_frac": round(bbytes / (bms * 1e-3) / 1e9 / peak, 4)}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a, g, src, st)

    line = {"metric": metric_name(a.workload, a.scale), "value": round(value, 3), "unit": unit,
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_max, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if a.workload == "pagerank" else ("u32" if weights else "i32"),
            "data": "synthetic (seeded RMAT, generated on the device)",
            "config": workload_config(a, V, E, src, {
                "iterations": st.iterations, "vertices_reached": st.vertices_reached,
                "edges_traversed": st.edges_traversed, "edges_relaxed": st.edges_relaxed}),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk}
    line.update(extra)
    g.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_baseline(a, g, src, st):
    """The oracle (CPU restatement of the reference's algorithm) on a bounded
    sample of the same workload, one host core."""
    from oracle import oracle
    rp, cl, w = g.csr()
    if a.workload == "sssp":
        _, edges, secs, settled = oracle.dijkstra(rp, cl, w, src, a.cpu_seconds)
        done = settled == st.vertices_reached
        return {"value": round(edges / secs / 1e9, 5), "unit": "GTEPS", "cores": 1,
                "kind": "port",
                "sample": f"serial binary-heap Dijkstra from the same source "
                          f"({'complete' if done else 'stopped after %.0f s' % a.cpu_seconds}, "
                          f"{settled} vertices settled, {edges} edges scanned, {secs:.2f} s); "
                          f"the reference has no CPU SSSP"}
    if a.workload == "bfs":
        edges, secs, reached = oracle.bfs_timed(rp, cl, src, a.cpu_seconds)
        return {"value": round(edges / secs / 1e9, 5), "unit": "GTEPS", "cores": 1,
                "kind": "port",
                "sample": f"restatement of testBFS.cu:64-79 (queue BFS), full traversal of the "
                          f"same graph and source ({reached} vertices, {secs:.3f} s)"}
    it = 3
    t = time.perf_counter()
    oracle.pagerank(rp, cl, 0.85, it, 0.0)
    secs = time.perf_counter() - t
    return {"value": round(len(cl) * it / secs / 1e9, 5), "unit": "GE/s/iter", "cores": 1,
            "kind": "port",
            "sample": f"FP64 PageRank restating testPageRank.cu:74-104 (plus dangling "
                      f"redistribution), {it} iterations on the same graph, {secs:.2f} s"}


# ------------------------------------------------------------ reference --
def run_reference(a, rank, world):
    if rank != 0:
        return
    from oracle import oracle
    threads = oracle.max_threads()
    rp, cl = oracle.rmat_csr_par(a.scale, 16, a.seed, threads)
    V, E = len(rp) - 1, len(cl)
    src = int(np.argmax(np.diff(rp.astype(np.int64))))
    bound = 8.0
    vals, ms = [], []
    if a.workload == "sssp":
        w = oracle.uint_weights_par(E, 2, 1, 255, threads)
        desc = (f"CPU restatement of SSSP.cu's frontier Bellman-Ford (edgeFilter atomicMin + "
                f"vertexFilter supersteps, oliver.h:56-113) on {threads} OpenMP threads; each "
                f"step a full solve or stopped after {bound:.0f} s; value = edges scanned / s")
        for i in range(a.warmup + a.steps):
            _, edges, secs, rounds = oracle.sssp_frontier(rp, cl, w, src, threads, bound)
            if i >= a.warmup:
                vals.append(edges / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "GTEPS", threads
    elif a.workload == "bfs":
        desc = ("restatement of testBFS.cu:64-79 (the reference's serial queue BFS; 1 core); "
                f"each step a full traversal or stopped after {bound:.0f} s")
        for i in range(a.warmup + a.steps):
            edges, secs, _ = oracle.bfs_timed(rp, cl, src, bound)
            if i >= a.warmup:
                vals.append(edges / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "GTEPS", 1
    else:
        desc = ("restatement of testPageRank.cu:74-104 (serial FP64 push PageRank, plus "
                "dangling redistribution; 1 core); each step 2 iterations")
        for i in range(a.warmup + a.steps):
            t = time.perf_counter()
            oracle.pagerank(rp, cl, 0.85, 2, 0.0)
            secs = time.perf_counter() - t
            if i >= a.warmup:
                vals.append(E * 2 / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "GE/s/iter", 1
    value = float(np.median(vals)) if vals else 0.0
    line = {"impl": "reference", "metric": metric_name(a.workload, a.scale),
            "value": round(value, 5), "unit": unit, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(float(np.median(ms)) if ms else 0.0, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if a.workload == "pagerank" else "u32",
            "data": "synthetic (seeded RMAT, generated on the host)",
            "config": workload_config(a, V, E, src),
            "cpu_baseline": {"value": round(value, 5), "unit": unit, "cores": cores,
                             "kind": "port", "sample": desc},
            "e2e": {"value": round(value, 5), "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", a.gpus if a.gpus == 1 else 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        run_reference(a, rank, world)
    else:
        run_ours(a, rank, world, local_rank)


if __name__ == "__main__":
    main()
