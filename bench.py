#!/usr/bin/env python
"""Benchmark of the olive_b200 frontier engine on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sssp|bfs|pagerank|msbfs|wpr|batch] [--scale S]

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
testBFS.cu's queue BFS (once per source for msbfs), or of testPageRank.cu's
FP64 PageRank, on the same synthetic graph built on the host; for wpr and
batch, which have no reference counterpart, the oracle's FP64 weighted
PageRank and BFS + PPR-32 per instance on the same inputs.  Each step's
sample is bounded by --ref-seconds.
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
    ap.add_argument("--workload", choices=["sssp", "bfs", "pagerank", "msbfs", "wpr", "batch"],
                    default="sssp")
    ap.add_argument("--scale", type=int, default=None)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="bound of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-seconds", type=float, default=8.0,
                    help="--impl reference: bound of one step's CPU sample")
    a = ap.parse_args()
    if a.scale is None:
        a.scale = {"pagerank": 22, "wpr": 20, "batch": 0}.get(a.workload, 24)
    a.warmup = max(a.warmup, 3) if a.impl == "ours" else a.warmup
    return a


def metric_name(w, scale):
    if w == "sssp":
        return f"SSSP GTEPS, RMAT-{scale} ef16, uint32 weights U[1,255], src = max out-degree"
    if w == "bfs":
        return f"BFS GTEPS, RMAT-{scale} ef16, src = max out-degree"
    if w == "msbfs":
        return (f"64-source BFS aggregate GTEPS, RMAT-{scale} ef16, sources uniform over "
                f"out-degree >= 1")
    if w == "wpr":
        return (f"weighted PageRank forward GE/s/iter, RMAT-{scale} ef16, lognormal FP32 weights; "
                f"forward+adjoint time reported against forward time")
    if w == "batch":
        return ("512 ER graphs (V in [1K,64K], 8 edges/vertex) block-diagonal: BFS + K=32 PPR "
                "per graph in one persistent launch, edge visits per second")
    return f"PageRank GE/s/iter, RMAT-{scale} ef16, alpha 0.85, FP32, dangling redistributed"


def workload_config(a, V=None, E=None, src=None, extra=None):
    c = {"workload": f"{a.workload}-rmat{a.scale}", "scale": a.scale, "edge_factor": 16,
         "rmat_abcd": [0.57, 0.19, 0.19, 0.05], "seed": a.seed, "V": V, "E": E,
         "parallelism": f"replicas x{a.gpus} (one whole graph per GPU)"}
    if a.workload == "sssp":
        c.update(weights="uint32 U[1,255], wseed 2", source=src)
    elif a.workload == "bfs":
        c.update(source=src)
    elif a.workload == "msbfs":
        c.update(sources="64 distinct, uniform over out-degree >= 1 (numpy seed 4)",
                 output="int32 levels [64][V]")
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


# Committed ncu launch-list summaries (profiles/*.md) of each default workload:
# their `traffic_bytes` line is the DRAM read + write of one solve as the
# profiler measured it (sum over the solve's launches; ncu flushes the caches
# before each launch, so this is a cold-cache upper bound of the warm run).
PROFILE_OF = {("sssp", 24): "sssp_rmat24.md", ("bfs", 24): "bfs_rmat24.md",
              ("pagerank", 22): "pagerank_rmat22.md", ("msbfs", 24): "msbfs_rmat24.md",
              ("wpr", 20): "wpr_rmat20.md", ("batch", 0): "batch_er512.md"}


def profile_traffic(workload, scale, seed, key="traffic_bytes"):
    """(bytes, source) from the committed profile summary of this workload
    (default size, seed 1), or (None, None)."""
    name = PROFILE_OF.get((workload, scale)) if seed == 1 else None
    path = os.path.join(ROOT, "profiles", name) if name else None
    if not path or not os.path.exists(path):
        return None, None
    for line in open(path):
        if line.startswith(key + ":"):
            return int(float(line.split(":", 1)[1].split()[0])), (
                f"profiles/{name} ({key}: ncu launch list, cold cache per launch)")
    return None, None


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
    if a.workload == "msbfs":
        rp, _, _ = g.csr()
        deg = np.diff(rp.astype(np.int64))
        srcs_np = np.random.default_rng(4).choice(np.flatnonzero(deg > 0), 64,
                                                 replace=False).astype(np.uint32)
        srcs = torch.from_numpy(srcs_np.astype(np.int32)).cuda()
        src = srcs_np.tolist()
        out = torch.empty((64, V), dtype=torch.int32, device="cuda")
    else:
        out = torch.empty(V, dtype=torch.float32 if a.workload == "pagerank" else torch.int32,
                          device="cuda")

    def step(dst):
        if a.workload == "sssp":
            return g.sssp(src, out=dst)
        if a.workload == "bfs":
            return g.bfs(src, out=dst)
        if a.workload == "msbfs":
            return g.msbfs(srcs, out=dst)
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
    elif a.workload == "msbfs":
        units = st.edges_traversed
        value = world * units / (ms_max * 1e-3) / 1e9
        unit = "GTEPS"
        alg_bytes = 4 * 64 * V + 12 * E + 24 * V * st.iterations
        bytes_formula = ("4 B per output level (64 x V) + 12 B/edge (one pass: index + "
                         "64-bit mask) + 24 B/vertex/level (visit, cur, next masks)")
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
    traffic, traffic_src = profile_traffic(a.workload, a.scale, a.seed)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "traffic_source": traffic_src,
                "kernel": f"whole {a.workload} solve (all kernels of one call, CUDA graph)",
                "algorithmic_bytes": int(alg_bytes), "bytes_formula": bytes_formula,
                "peak_source": peak_src, "kernel_ms": round(kern_ms, 4)}

    # launches of our kernels per step (kernel nodes executed by the graph):
    # sssp: fill, init, 4 per superstep, the map back to the caller's ids
    # (renumbered run), reached count; bfs: fill, init, 9 per level
    if a.workload == "sssp":
        per_step = 2 + 4 * st.iterations + 1 + int(g.tune().get("sssp_relabel", 0))
    elif a.workload == "bfs":
        per_step = 2 + 9 * st.iterations
    elif a.workload == "msbfs":
        per_step = 2 + 6 * st.iterations + 1
    else:   # pagerank: segments (when the graph has long rows), blocks, fold per iteration
        per_step = 2 + 3 * st.iterations
    launches = per_step * a.steps

    # end to end through the public API: host (pinned) output buffer, D2H inside
    host_out = torch.empty(out.shape, dtype=out.dtype, pin_memory=True)
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
           "h2d_bytes_per_step": 256 if a.workload == "msbfs" else 0,
           "d2h_bytes_per_step": int(out.numel() * 4),
           "ms_per_step": round(e2e_ms, 4),
           "note": "olv_* call with a pinned host output buffer; the per-call input is the "
                   "source id passed by value; graph resident as after Oliver::readGraph"}

    extra = {}
    if a.workload == "msbfs":
        # the same 64 sources as 64 sequential plain BFS runs
        lv = torch.empty(V, dtype=torch.int32, device="cuda")
        for s0 in src[:3]:
            g.bfs(s0, out=lv)
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        q0.record(stream)
        seq_edges = 0
        for s0 in src:
            g.bfs(s0, out=lv)
            seq_edges += g.last_stats.edges_traversed
        q1.record(stream)
        torch.cuda.synchronize()
        seq_ms = q0.elapsed_time(q1)
        seq_gteps = seq_edges / (seq_ms * 1e-3) / 1e9
        extra["sequential_plain"] = {"value": round(seq_gteps, 3), "unit": "GTEPS",
                                     "ms_for_64": round(seq_ms, 3),
                                     "speedup_of_batched": round(value / world / seq_gteps, 2)}
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
    if a.workload == "msbfs":
        edges, secs, runs = 0, 0.0, 0
        for s0 in src:
            e, t, _ = oracle.bfs_timed(rp, cl, s0, a.cpu_seconds)
            edges += e
            secs += t
            runs += 1
            if secs > a.cpu_seconds:
                break
        return {"value": round(edges / secs / 1e9, 5), "unit": "GTEPS", "cores": 1,
                "kind": "port",
                "sample": f"restatement of testBFS.cu:64-79 run sequentially for the first "
                          f"{runs} of the 64 sources ({secs:.2f} s)"}
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


def common_line(a, world, metric_unit, value, ms, dtype, data, config, roofline, cpu, e2e,
                launches, clk, extra):
    line = {"metric": metric_name(a.workload, a.scale), "value": round(value, 3),
            "unit": metric_unit, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": data, "config": config,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk}
    line.update(extra)
    return line


def timed(stream, fn, steps):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def max_over_ranks(x, world):
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_wpr(a, rank, world, local_rank):
    """Weighted PageRank forward + adjoint on RMAT-20 (lognormal FP32 weights,
    Dirichlet(1) personalisation, g ~ N(0,1)); a step is one forward and one
    backward solve of 100 sweeps each."""
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    import olive_b200 as ob
    stream = torch.cuda.current_stream()
    g = ob.Graph.rmat(a.scale, 16, a.seed)
    g.set_stream(stream)
    V, E = g.V, g.E
    rng = np.random.default_rng(7)
    w = torch.from_numpy(rng.lognormal(0.0, 1.0, E).astype(np.float32)).cuda()
    pn = rng.exponential(1.0, V)
    p = torch.from_numpy((pn / pn.sum()).astype(np.float32)).cuda()
    gv = torch.from_numpy(rng.standard_normal(V).astype(np.float32)).cuda()
    r = torch.empty(V, dtype=torch.float32, device="cuda")
    dw = torch.empty(E, dtype=torch.float32, device="cuda")
    dp = torch.empty(V, dtype=torch.float32, device="cuda")
    it = 100
    g.wpr_forward(p, w=w, max_it=it, out=r)

    def fwd():
        g.wpr_forward(p, max_it=it, out=r)

    def bwd():
        g.wpr_backward(gv, max_it=it, dw_out=dw, dp_out=dp)

    for _ in range(a.warmup):
        fwd()
        bwd()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    ms_f = max_over_ranks(timed(stream, fwd, a.steps), world)
    ms_b = max_over_ranks(timed(stream, bwd, a.steps), world)
    clk = clocks.stop()
    fs = g.last_stats
    units = E * it
    value = world * units / (ms_f * 1e-3) / 1e9
    peak, peak_src = peaks()
    alg = (12 * E + 20 * V) * it
    traffic, traffic_src = profile_traffic("wpr", a.scale, a.seed, "traffic_bytes_forward")
    roofline = {"bound": "hbm", "achieved": round(alg / (ms_f * 1e-3) / 1e9, 1), "peak": peak,
                "unit": "GB/s", "frac": round(alg / (ms_f * 1e-3) / 1e9 / peak, 4),
                "traffic": traffic, "traffic_source": traffic_src,
                "kernel": "forward solve (100 pull sweeps, CUDA graph)",
                "algorithmic_bytes": int(alg),
                "bytes_formula": "(12 B/edge: CSC index, weight, r/W gather + 20 B/vertex) per sweep",
                "peak_source": peak_src}
    host_dw = torch.empty(E, dtype=torch.float32, pin_memory=True)
    host_dp = torch.empty(V, dtype=torch.float32, pin_memory=True)
    host_r = torch.empty(V, dtype=torch.float32, pin_memory=True)
    host_p = p.cpu().pin_memory()
    host_g = gv.cpu().pin_memory()

    def e2e_step():
        g.wpr_forward(host_p, max_it=it, out=host_r)
        g.wpr_backward(host_g, max_it=it, dw_out=host_dw, dp_out=host_dp)

    t0 = time.perf_counter()
    for _ in range(a.steps):
        e2e_step()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / a.steps, world)
    e2e = {"value": round(world * units / (e2e_ms * 1e-3) / 1e9, 3), "unit": "GE/s/iter",
           "h2d_bytes_per_step": 8 * V, "d2h_bytes_per_step": 4 * (E + 2 * V),
           "ms_per_step": round(e2e_ms, 3),
           "note": "forward + backward through olv_wpr_* with pinned host p, g, r, dw, dp"}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        from oracle import oracle
        rp, cl, _ = g.csr()
        w64 = w.double().cpu().numpy()
        t = time.perf_counter()
        rr = oracle.wpr_forward(rp, cl, w64, p.double().cpu().numpy(), 0.85, 3)
        secs = time.perf_counter() - t
        cpu = {"value": round(E * 3 / secs / 1e9, 5), "unit": "GE/s/iter", "cores": 1,
               "kind": "port", "sample": f"FP64 weighted PageRank forward (oracle), 3 sweeps, "
                                         f"{secs:.2f} s"}
    launches = (2 + 3 * it) + (5 + 3 * it)
    config = workload_config(a, V, E, None, {
        "weights": "lognormal(0,1) FP32, numpy seed 7", "p": "Dirichlet(1)", "g": "N(0,1)",
        "alpha": 0.85, "sweeps": it, "forward_ms": round(ms_f, 3), "backward_ms": round(ms_b, 3)})
    extra = {"fwd_bwd_over_fwd": round((ms_f + ms_b) / ms_f, 3),
             "target": "forward+adjoint <= 3x forward"}
    line = common_line(a, world, "GE/s/iter", value, ms_f + ms_b, "f32",
                       "synthetic (seeded RMAT on the device, numpy weights)", config, roofline,
                       cpu, e2e, launches * a.steps, clk, extra)
    g.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batch(a, rank, world, local_rank):
    """512 ER digraphs packed block-diagonally; a step is one persistent launch
    running BFS from local vertex 0 and K=32 PPR vectors (max 50 iterations,
    tol 1e-7) for every graph."""
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    import olive_b200 as ob
    stream = torch.cuda.current_stream()
    count, K = 512, 32
    g, off = ob.Graph.er_batch(count, 1024, 65536, 8, seed=a.seed)
    g.set_stream(stream)
    V, E = g.V, g.E
    n = np.diff(off.astype(np.int64))
    rng = np.random.default_rng(11)
    seeds = np.stack([rng.integers(0, ni, K) for ni in n]).astype(np.uint32)
    lv = torch.empty(V, dtype=torch.int32, device="cuda")
    pr = torch.empty((V, K), dtype=torch.float32, device="cuda")

    def step():
        g.batch(off, seeds, K=K, alpha=0.85, max_it=50, tol=1e-7, levels_out=lv, ppr_out=pr)

    for _ in range(a.warmup):
        step()
    st = g.last_stats
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    ms = max_over_ranks(timed(stream, step, a.steps), world)
    clk = clocks.stop()
    st = g.last_stats
    visits = st.edges_traversed + st.edges_relaxed      # BFS edges + PPR edge-vectors
    value = world * visits / (ms * 1e-3) / 1e9
    peak, peak_src = peaks()
    _, _, iters = g.batch(off, seeds, K=K, max_it=50, tol=1e-7, levels_out=lv, ppr_out=pr)
    alg = 8 * st.edges_traversed + 4 * st.edges_relaxed + (4 + 8 * K) * V * 1
    traffic, traffic_src = profile_traffic("batch", a.scale, a.seed)
    roofline = {"bound": "hbm", "achieved": round(alg / (ms * 1e-3) / 1e9, 1), "peak": peak,
                "unit": "GB/s", "frac": round(alg / (ms * 1e-3) / 1e9 / peak, 4),
                "traffic": traffic, "traffic_source": traffic_src,
                "kernel": "k_batch (one persistent launch)", "algorithmic_bytes": int(alg),
                "bytes_formula": "8 B/BFS edge + 4 B per PPR edge-vector visit (128 B row per "
                                 "in-edge for K=32) + (4 + 8K) B/vertex"}
    host_lv = torch.empty(V, dtype=torch.int32, pin_memory=True)
    host_pr = torch.empty((V, K), dtype=torch.float32, pin_memory=True)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        g.batch(off, seeds, K=K, max_it=50, tol=1e-7, levels_out=host_lv, ppr_out=host_pr)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / a.steps, world)
    e2e = {"value": round(world * visits / (e2e_ms * 1e-3) / 1e9, 3), "unit": "G visits/s",
           "h2d_bytes_per_step": int(4 * (count + 1) + seeds.nbytes),
           "d2h_bytes_per_step": int(4 * V * (1 + K)), "ms_per_step": round(e2e_ms, 3)}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        from oracle import oracle
        rp, cl, _ = g.csr()
        t = time.perf_counter()
        done, cvis = 0, 0
        for i in range(count):
            b0, b1 = int(off[i]), int(off[i + 1])
            lrp = (rp[b0:b1 + 1] - rp[b0]).astype(np.uint32)
            lcl = (cl[rp[b0]:rp[b1]] - b0).astype(np.uint32)
            _, e = oracle.bfs(lrp, lcl, 0)
            _, itn = oracle.ppr(lrp, lcl, seeds[i], 0.85, 50, 1e-7)
            cvis += e + itn * len(lcl) * K
            done += 1
            if time.perf_counter() - t > a.cpu_seconds:
                break
        secs = time.perf_counter() - t
        cpu = {"value": round(cvis / secs / 1e9, 5), "unit": "G visits/s", "cores": 1,
               "kind": "port", "sample": f"oracle BFS + FP64 PPR-32 per instance, first {done} "
                                         f"of {count} instances, {secs:.1f} s"}
    config = {"workload": "batch-er512", "instances": count, "V_range": [1024, 65536],
              "avg_degree": 8, "K": K, "alpha": 0.85, "max_it": 50, "tol": 1e-7,
              "seed": a.seed, "V": V, "E": E, "ppr_iterations_mean": float(np.mean(iters)),
              "parallelism": f"replicas x{world}",
              "l2": "inputs larger than L2 (PPR state 2 x V x 128 B = 4.3 GB)"}
    line = common_line(a, world, "G visits/s", value, ms, "f32+i32",
                       "synthetic (seeded ER batch generated on the host)", config, roofline,
                       cpu, e2e, a.steps, clk, {})
    g.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------ reference --
def run_reference(a, rank, world):
    if rank != 0:
        return
    from oracle import oracle
    threads = oracle.max_threads()
    bound = a.ref_seconds
    vals, ms = [], []
    if a.workload == "batch":
        # the same 512 ER instances and PPR seeds as the GPU arm (the oracle's
        # restatement of the batch generator), BFS from local vertex 0 plus
        # PPR-32 per instance, instances in order until the bound
        count, K = 512, 32
        sizes = oracle.er_batch_sizes(count, 1024, 65536, a.seed)
        rng = np.random.default_rng(11)
        seeds = [rng.integers(0, ni, K).astype(np.uint32) for ni in sizes]
        V, E = int(sizes.sum()), int(8 * sizes.sum())
        desc = (f"oracle BFS + FP64 PPR-{K} per instance (serial, 1 core), instances in "
                f"order; each step stopped after {bound:.0f} s; value = edge visits / s")
        for i in range(a.warmup + a.steps):
            visits, secs = 0, 0.0
            for j in range(count):
                lrp, lcl = oracle.er_batch_instance(j, int(sizes[j]), 8, a.seed)
                t = time.perf_counter()
                _, e = oracle.bfs(lrp, lcl, 0)
                _, itn = oracle.ppr(lrp, lcl, seeds[j], 0.85, 50, 1e-7)
                secs += time.perf_counter() - t
                visits += e + itn * len(lcl) * K
                if secs > bound:
                    break
            if i >= a.warmup:
                vals.append(visits / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "G visits/s", 1
        line = {"impl": "reference", "metric": metric_name(a.workload, a.scale),
                "value": round(float(np.median(vals)) if vals else 0.0, 5), "unit": unit,
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": round(float(np.median(ms)) if ms else 0.0, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64+i32", "data": "synthetic (seeded ER batch generated on the host)",
                "config": {"workload": "batch-er512", "instances": count,
                           "V_range": [1024, 65536], "avg_degree": 8, "K": K, "alpha": 0.85,
                           "max_it": 50, "tol": 1e-7, "seed": a.seed, "V": V, "E": E}}
        line["cpu_baseline"] = {"value": line["value"], "unit": unit, "cores": cores,
                                "kind": "port", "sample": desc}
        line["e2e"] = {"value": line["value"], "unit": unit, "h2d_bytes_per_step": 0,
                       "d2h_bytes_per_step": 0}
        print(json.dumps(line), flush=True)
        return
    rp, cl = oracle.rmat_csr_par(a.scale, 16, a.seed, threads)
    V, E = len(rp) - 1, len(cl)
    src = int(np.argmax(np.diff(rp.astype(np.int64))))
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
    elif a.workload == "msbfs":
        deg = np.diff(rp.astype(np.int64))
        srcs = np.random.default_rng(4).choice(np.flatnonzero(deg > 0), 64, replace=False)
        desc = ("restatement of testBFS.cu:64-79 (serial queue BFS, 1 core) run once per source; "
                f"each step the 64 sources in turn, stopped after {bound:.0f} s")
        for i in range(a.warmup + a.steps):
            edges, secs = 0, 0.0
            for s0 in srcs:
                e, t, _ = oracle.bfs_timed(rp, cl, int(s0), bound)
                edges += e
                secs += t
                if secs > bound:
                    break
            if i >= a.warmup:
                vals.append(edges / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "GTEPS", 1
    elif a.workload == "bfs":
        desc = ("restatement of testBFS.cu:64-79 (the reference's serial queue BFS; 1 core); "
                f"each step a full traversal or stopped after {bound:.0f} s")
        for i in range(a.warmup + a.steps):
            edges, secs, _ = oracle.bfs_timed(rp, cl, src, bound)
            if i >= a.warmup:
                vals.append(edges / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "GTEPS", 1
    elif a.workload == "wpr":
        # the GPU arm's inputs: lognormal weights and Dirichlet(1) p, numpy seed 7
        rng = np.random.default_rng(7)
        w = rng.lognormal(0.0, 1.0, E).astype(np.float32).astype(np.float64)
        pn = rng.exponential(1.0, V)
        p = (pn / pn.sum()).astype(np.float32).astype(np.float64)
        desc = ("oracle FP64 weighted PageRank forward (the reference has no weighted PR; "
                "1 core); each step 2 sweeps")
        for i in range(a.warmup + a.steps):
            t = time.perf_counter()
            oracle.wpr_forward(rp, cl, w, p, 0.85, 2)
            secs = time.perf_counter() - t
            if i >= a.warmup:
                vals.append(E * 2 / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "GE/s/iter", 1
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
            "dtype": "f64" if a.workload in ("pagerank", "wpr") else "u32",
            "data": "synthetic (seeded RMAT, generated on the host)",
            "config": workload_config(a, V, E, src, {
                "weights": "lognormal(0,1) FP32, numpy seed 7", "p": "Dirichlet(1)",
                "sweeps_per_step": 2} if a.workload == "wpr" else None),
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
    elif a.workload == "wpr":
        run_wpr(a, rank, world, local_rank)
    elif a.workload == "batch":
        run_batch(a, rank, world, local_rank)
    else:
        run_ours(a, rank, world, local_rank)


if __name__ == "__main__":
    main()
