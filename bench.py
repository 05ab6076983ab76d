#!/usr/bin/env python
"""Benchmark of the olive_b200 frontier engine on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sssp|bfs|pagerank|msbfs|wpr|batch] [--scale S]
                    [--no-extras] [--no-parity]

Default workload: single-source shortest paths (frontier Bellman-Ford with
atomicMin, SSSP.cu semantics) on an RMAT graph of scale 24, edge factor 16,
(a,b,c,d) = (.57,.19,.19,.05), uint32 weights uniform in [1,255], from the
highest out-degree vertex.  A step is one complete solve on the resident
graph.  The metric is GTEPS = (sum of out-degrees of reached vertices) / time.
The default line also carries, as extra keys, BFS on the same graph ("bfs"),
64-source BFS on RMAT-24 ("msbfs"), PageRank on RMAT-22 ("pagerank"), 32
personalised PageRank vectors on RMAT-22 ("ppr"), weighted PageRank forward +
adjoint on RMAT-20 ("wpr") and the 512-graph ER batch ("batch"), each with its
own timing, roofline fraction and parity check; a caller arriving with a host
CSR ("e2e_cold": graph upload and build + one solve + the result read back);
the GPU text writer against the host printf loop ("writer"); and the
reference's BFS.cu compiled unmodified against the header layer, plus the
same loop with the pull opt-ins, on the same graph ("dropin_bfs").

Parity: every line checks the GPU result of its last step against the CPU
oracle on rank 0 ("parity" key): SSSP against a complete serial Dijkstra,
BFS against the restated testBFS queue BFS, msBFS rows against 64 solo GPU
runs and the oracle, PageRank / weighted PageRank against the FP64 oracle
after the same iterations, the batch against per-instance oracle runs.

One process per GPU (torchrun); every rank runs its own replica of the
workload (the traversal does not shard: "replicas only"), `value` sums the
ranks' work over the slowest rank's time.  Rank 0 prints one JSON line.

--impl reference times the reference's algorithm on the host cores:
* sssp: the CPU restatement of SSSP.cu's frontier Bellman-Ford on all host
  threads (the reference has no CPU SSSP), value = E_reached / t as for the
  GPU arm (edges scanned, which include re-relaxations, reported beside it);
* bfs: the reference's own testBFS binary (oracle/_ref, built unmodified from
  the reference sources) on a written edge-list file up to scale 22; above
  that (the text file passes 3 GB) the restatement of testBFS.cu:64-79;
* pagerank: the reference's own testPageRank binary with -max 50 (its loop
  timer; the file parse is excluded);
* msbfs: the testBFS restatement once per source;
* wpr, batch (no reference counterpart): the oracle's FP64 weighted PageRank
  and BFS + PPR-32 per instance on the same inputs.
Each step's sample is bounded by --ref-seconds (the reference binaries run as
many whole solves as fit in about two minutes).
"""
import argparse
import copy
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
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
    ap.add_argument("--workload", choices=["sssp", "bfs", "pagerank", "msbfs", "wpr", "batch",
                                           "ppr"], default="sssp")
    ap.add_argument("--scale", type=int, default=None)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="bound of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the msbfs/pagerank/wpr/batch extra keys")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle comparison")
    ap.add_argument("--ref-seconds", type=float, default=8.0,
                    help="--impl reference: bound of one step's CPU sample")
    a = ap.parse_args()
    if a.scale is None:
        a.scale = default_scale(a.workload)
    a.warmup = max(a.warmup, 3) if a.impl == "ours" else a.warmup
    return a


def default_scale(w):
    return {"pagerank": 22, "ppr": 22, "wpr": 20, "batch": 0}.get(w, 24)


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
    if w == "ppr":
        return (f"K=32 personalised PageRank GE/s/iter (edge visits carrying 32 values), "
                f"RMAT-{scale} ef16, alpha 0.85, FP32")
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
# profiler measured it (see each file for how it was taken and scaled).
PROFILE_OF = {("sssp", 24): "sssp_rmat24.md", ("bfs", 24): "bfs_rmat24.md",
              ("pagerank", 22): "pagerank_rmat22.md", ("msbfs", 24): "msbfs_rmat24.md",
              ("wpr", 20): "wpr_rmat20.md", ("batch", 0): "batch_er512.md",
              ("ppr", 22): "ppr_rmat22.md"}


def profile_traffic(workload, scale, seed, key="traffic_bytes"):
    """(bytes, source) from the committed profile summary of this workload
    (default size, seed 1), or (None, None)."""
    name = PROFILE_OF.get((workload, scale)) if seed == 1 else None
    path = os.path.join(ROOT, "profiles", name) if name else None
    if not path or not os.path.exists(path):
        return None, None
    for line in open(path):
        if line.startswith(key + ":"):
            return int(float(line.split(":", 1)[1].split()[0])), f"profiles/{name} ({key})"
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
        time.sleep(0.3)   # let the sampler start before the timed region

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


# ------------------------------------------------------------- helpers --
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


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


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


def rel_err(got, ref):
    got = np.asarray(got, np.float64)
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300))) if len(ref) else 0.0


# ------------------------------------------------------------- parity --
def parity_exact(got, ref, vs):
    got = np.asarray(got).view(np.uint32)
    ref = np.asarray(ref).view(np.uint32)
    mism = int(np.count_nonzero(got != ref))
    return {"checked": True, "vs": vs, "compared": int(len(ref)), "mismatches": mism,
            "pass": mism == 0}


def parity_float(err, tol, vs, extra=None):
    d = {"checked": True, "vs": vs, "max_rel_err": err, "tolerance": tol, "pass": err < tol}
    if extra:
        d.update(extra)
    return d


def cold_e2e(ob, stream, rp, cl, w, src, method, reps=2):
    """A caller that arrives with a host CSR: olv_graph_create (upload, reverse
    graph built on the device), then the first solve into a pinned host
    buffer, then olv_graph_destroy -- all inside the wall-clock region."""
    import torch
    rp_p = torch.from_numpy(rp.view(np.int32)).pin_memory()
    cl_p = torch.from_numpy(cl.view(np.int32)).pin_memory()
    w_p = None if w is None else torch.from_numpy(w.view(np.int32)).pin_memory()
    host = torch.empty(len(rp) - 1, dtype=torch.int32, pin_memory=True)
    best = None
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        # int32 tensors carry the uint32 bits; integer weights become OLV_W_U32
        g = ob.Graph.from_csr(rp_p, cl_p) if w is None else ob.Graph.from_csr(rp_p, cl_p, w_p)
        g.set_stream(stream)
        getattr(g, method)(src, out=host)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        st = g.last_stats
        g.close()
        best = ms if best is None else min(best, ms)
    h2d = rp.nbytes + cl.nbytes + (0 if w is None else w.nbytes)
    return {"value": round(st.edges_traversed / (best * 1e-3) / 1e9, 3), "unit": "GTEPS",
            "ms": round(best, 2), "h2d_bytes": int(h2d), "d2h_bytes": int(4 * (len(rp) - 1)),
            "note": "host CSR in pinned memory -> olv_graph_create (upload + reverse graph on "
                    "the device) -> first solve (per-graph structures built) -> pinned host "
                    "result -> olv_graph_destroy; wall clock, best of %d" % reps}


def writer_line(ob, dev_vals, stream):
    """The solve's V results written as "%d\\n" text from device memory
    (olv_write_text: formatted on the GPU, one fwrite per 2^24 values) against
    the reference's way (a host fprintf per vertex), both to local files,
    which must be identical."""
    import torch
    from oracle import oracle
    work = tempfile.mkdtemp(prefix="olv_writer_")
    a, b = os.path.join(work, "gpu.txt"), os.path.join(work, "printf.txt")
    vals = dev_vals.view(torch.int32)
    ob.write_text(a, vals, stream)               # warm-up (allocations)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nbytes = ob.write_text(a, vals, stream)
    gpu_s = time.perf_counter() - t0
    host = vals.cpu().numpy()
    cpu_s = oracle.fprintf_i32(b, host)
    same = open(a, "rb").read() == open(b, "rb").read()
    shutil.rmtree(work, ignore_errors=True)
    return {"values": int(vals.numel()), "bytes": int(nbytes), "gpu_ms": round(gpu_s * 1e3, 2),
            "gpu_GB_per_s": round(nbytes / gpu_s / 1e9, 3),
            "printf_loop_ms": round(cpu_s * 1e3, 2), "speedup": round(cpu_s / gpu_s, 2),
            "identical_bytes": bool(same),
            "note": "olv_write_text from device memory to a local file (format on the GPU, "
                    "D2H, fwrite) vs one fprintf per value on one host core"}


def dropin_line(g, src, lv_dev, bfs_c_abi):
    """The reference's BFS.cu compiled unmodified against the header layer
    (olive_b200/_apps/BFS) and the same loop with the pull opt-ins
    (olive_b200/_apps/BFSPullOptIn), on this graph written as a binary CSR
    file, timed by the apps' own clock (their loop, as BFS.cu:150-151 logs
    it), levels checked against olv_bfs."""
    apps = os.path.join(ROOT, "olive_b200", "_apps")
    if not os.path.exists(os.path.join(apps, "BFS")):
        return {"unavailable": "olive_b200/_apps/BFS not built (needs the reference sources at "
                               "build time)"}
    work = tempfile.mkdtemp(prefix="olv_dropin_")
    path = os.path.join(work, "g.bin")
    g.save(path)
    want = lv_dev.cpu().numpy().astype(np.int64)
    e_reached = bfs_c_abi["value"] * bfs_c_abi["ms"] * 1e6
    out = {"graph": "the SSSP line's RMAT-24 as a binary CSR file", "source": int(src),
           "olv_bfs_ms": bfs_c_abi["ms"]}
    for name in ("BFS", "BFSPullOptIn"):
        best = None
        for _ in range(2):
            p = subprocess.run([os.path.join(apps, name), path, "-s", str(src), "-round", "100000"],
                               cwd=work, capture_output=True, text=True, timeout=600)
            m = re.findall(r"iterations: (\d+), time: ([0-9.]+)ms", p.stderr + p.stdout)
            if p.returncode == 0 and m:
                t = float(m[-1][1])
                best = t if best is None else min(best, t)
        import pandas as pd
        got = pd.read_csv(os.path.join(work, "BFS.txt"), header=None, dtype=np.int64)[0].values
        key = "unmodified" if name == "BFS" else "pull_optin"
        out[key] = {"app": f"olive_b200/_apps/{name}", "ms": best,
                    "gteps": round(e_reached / (best * 1e-3) / 1e9, 2) if best else None,
                    "over_olv_bfs": round(best / bfs_c_abi["ms"], 2) if best else None,
                    "parity": {"vs": "olv_bfs levels", "mismatches": int(np.count_nonzero(got != want))}}
    shutil.rmtree(work, ignore_errors=True)
    out["note"] = ("app's own loop timer (frontier.size() host reads included, file load and "
                   "readGraph excluded); BFS.cu's functors cannot skip visited destinations, so its "
                   "levels are top-down over every frontier edge; the opt-in variant declares "
                   "pullCandidate / pullFirstHit")
    return out


# ------------------------------------------------- traversal workloads --
def traversal_line(a, rank, world, local_rank, extra_keys=True):
    """SSSP / BFS / msBFS / PageRank on a seeded RMAT graph built on the device."""
    import torch
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
    barrier(world)
    clocks = ClockSampler(local_rank)
    clocks.start()
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dev_ms = []
    for _ in range(a.steps):
        step(out)
        dev_ms.append(g.last_stats.device_ms)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1) / a.steps
    clk = clocks.stop()
    st = g.last_stats
    ms_max = max_over_ranks(ms, world)

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
    if traffic:
        roofline["traffic_over_algorithmic"] = round(traffic / alg_bytes, 3)

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
    e2e_ms = max_over_ranks(max(x0.elapsed_time(x1) / a.steps, wall_ms), world)
    e2e = {"value": round(world * units / (e2e_ms * 1e-3) / 1e9, 3), "unit": unit,
           "h2d_bytes_per_step": 256 if a.workload == "msbfs" else 0,
           "d2h_bytes_per_step": int(out.numel() * 4),
           "ms_per_step": round(e2e_ms, 4),
           "note": "olv_* call with a pinned host output buffer; the per-call input is the "
                   "source id passed by value; graph resident as after Oliver::readGraph"}

    extra = {}
    check = rank == 0 and not a.no_parity
    from oracle import oracle
    rp = cl = w = None
    if check or (rank == 0 and world == 1 and not a.no_cpu_baseline) or \
            (a.workload in ("sssp", "bfs") and extra_keys):
        rp, cl, w = g.csr()
    ref_info = None
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
                                     "speedup_of_batched": round(value / world / seq_gteps, 2),
                                     "target": ">= 10x"}
        if check:
            bad = 0
            for s, s0 in enumerate(src):
                g.bfs(s0, out=lv)
                bad += int(not torch.equal(out[s], lv))
            orows = [0, 63]
            obad = 0
            for s in orows:
                ref, _ = oracle.bfs(rp, cl, src[s])
                obad += int(np.count_nonzero(out[s].cpu().numpy() != ref))
            extra["parity"] = {"checked": True, "vs": "64 solo GPU BFS runs (every row) and "
                               "the oracle BFS (rows 0 and 63)", "rows_differing_from_solo": bad,
                               "oracle_mismatches": obad, "pass": bad == 0 and obad == 0}
    elif check and a.workload == "sssp":
        ref, e_ref, secs, nset = oracle.dijkstra(rp, cl, w, src)
        extra["parity"] = parity_exact(out.cpu().numpy(), ref,
                                       "serial binary-heap Dijkstra (complete)")
        ref_info = (e_ref, secs, nset)
    elif check and a.workload == "bfs":
        ref, _ = oracle.bfs(rp, cl, src)
        extra["parity"] = parity_exact(out.cpu().numpy(), ref, "testBFS.cu:64-79 restated")
    elif check:
        it = st.iterations
        ref, it_ref, _ = oracle.pagerank(rp, cl, 0.85, it, 0.0)
        extra["parity"] = parity_float(rel_err(out.cpu().numpy(), ref), 1e-6,
                                       f"FP64 oracle after the same {it} iterations")
    # BFS on the same graph, reported beside the SSSP headline
    if a.workload == "sssp" and extra_keys:
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
            "roofline_frac": round(bbytes / (bms * 1e-3) / 1e9 / peak, 4),
            "roofline_note": "8 B per edge of the reached set (a TEPS normalisation: the pull "
                             "levels stop at the first visited parent and read fewer edges)"}
        btraffic, _ = profile_traffic("bfs", a.scale, a.seed)
        if btraffic:
            extra["bfs"]["dram_frac"] = round(btraffic / (bms * 1e-3) / 1e9 / peak, 4)
            extra["bfs"]["dram_note"] = "profiled DRAM bytes of one solve / solve time / peak"
        if check:
            ref, _ = oracle.bfs(rp, cl, src)
            extra["bfs"]["parity"] = parity_exact(lv.cpu().numpy(), ref,
                                                  "testBFS.cu:64-79 restated")
    if a.workload in ("sssp", "bfs") and extra_keys and rank == 0:
        method = "sssp" if a.workload == "sssp" else "bfs"
        extra["e2e_cold"] = cold_e2e(ob, stream, rp, cl, w if weights else None, src, method)
        extra["writer"] = writer_line(ob, out, stream)
        if a.workload == "sssp":
            extra["dropin_bfs"] = dropin_line(g, src, lv, extra["bfs"])

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a, rp, cl, w, src, st, ref_info)

    config = workload_config(a, V, E, src, {
        "iterations": st.iterations, "vertices_reached": st.vertices_reached,
        "edges_traversed": st.edges_traversed, "edges_relaxed": st.edges_relaxed})
    dtype = "f32" if a.workload == "pagerank" else ("u32" if weights else "i32")
    line = common_line(a, world, unit, value, ms_max, dtype,
                       "synthetic (seeded RMAT, generated on the device)", config, roofline, cpu,
                       e2e, launches, clk, extra)
    g.close()
    return line


def cpu_baseline(a, rp, cl, w, src, st, ref_info=None):
    """The oracle (CPU restatement of the reference's algorithm) on a bounded
    sample of the same workload, one host core."""
    from oracle import oracle
    if a.workload == "sssp":
        if ref_info is not None:    # the complete Dijkstra the parity check already timed
            edges, secs, settled = ref_info
        else:
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


# ------------------------------------------------------ weighted PageRank --
def wpr_line(a, rank, world, local_rank):
    """Weighted PageRank forward + adjoint on RMAT-20 (lognormal FP32 weights,
    Dirichlet(1) personalisation, g ~ N(0,1)); a step is one forward and one
    backward solve of 100 sweeps each."""
    import torch
    import olive_b200 as ob
    stream = torch.cuda.current_stream()
    g = ob.Graph.rmat(a.scale, 16, a.seed)
    g.set_stream(stream)
    V, E = g.V, g.E
    rng = np.random.default_rng(7)
    w_np = rng.lognormal(0.0, 1.0, E).astype(np.float32)
    w = torch.from_numpy(w_np).cuda()
    pn = rng.exponential(1.0, V)
    p_np = (pn / pn.sum()).astype(np.float32)
    p = torch.from_numpy(p_np).cuda()
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
    barrier(world)
    ms_f = max_over_ranks(timed(stream, fwd, a.steps), world)
    ms_b = max_over_ranks(timed(stream, bwd, a.steps), world)
    clk = clocks.stop()
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
    extra = {"fwd_bwd_over_fwd": round((ms_f + ms_b) / ms_f, 3),
             "target": "forward+adjoint <= 3x forward"}
    from oracle import oracle
    rp = cl = None
    if rank == 0 and (not a.no_parity or (world == 1 and not a.no_cpu_baseline)):
        rp, cl, _ = g.csr()
    if rank == 0 and not a.no_parity:
        ref = oracle.wpr_forward(rp, cl, w_np.astype(np.float64), p_np.astype(np.float64), 0.85,
                                 it)
        extra["parity"] = parity_float(rel_err(host_r.numpy(), ref), 1e-5,
                                       f"FP64 oracle forward, {it} sweeps (per-vertex relative)")
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        t = time.perf_counter()
        oracle.wpr_forward(rp, cl, w_np.astype(np.float64), p_np.astype(np.float64), 0.85, 3)
        secs = time.perf_counter() - t
        cpu = {"value": round(E * 3 / secs / 1e9, 5), "unit": "GE/s/iter", "cores": 1,
               "kind": "port", "sample": f"FP64 weighted PageRank forward (oracle), 3 sweeps, "
                                         f"{secs:.2f} s"}
    launches = (2 + 3 * it) + (5 + 3 * it)
    config = workload_config(a, V, E, None, {
        "weights": "lognormal(0,1) FP32, numpy seed 7", "p": "Dirichlet(1)", "g": "N(0,1)",
        "alpha": 0.85, "sweeps": it, "forward_ms": round(ms_f, 3), "backward_ms": round(ms_b, 3)})
    line = common_line(a, world, "GE/s/iter", value, ms_f + ms_b, "f32",
                       "synthetic (seeded RMAT on the device, numpy weights)", config, roofline,
                       cpu, e2e, launches * a.steps, clk, extra)
    g.close()
    return line


# ---------------------------------------------------------------- batch --
def batch_line(a, rank, world, local_rank):
    """512 ER digraphs packed block-diagonally; a step is one persistent launch
    running BFS from local vertex 0 and K=32 PPR vectors (max 50 iterations,
    tol 1e-7) for every graph."""
    import torch
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
    clocks = ClockSampler(local_rank)
    clocks.start()
    barrier(world)
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
                                 "in-edge for K=32) + (4 + 8K) B/vertex",
                "note": "the PPR row gathers mostly hit L2 (the instances in flight fit it), so "
                        "the algorithmic bytes exceed the DRAM traffic"}
    if traffic:
        roofline["dram_frac"] = round(traffic / (ms * 1e-3) / 1e9 / peak, 4)
    host_lv = torch.empty(V, dtype=torch.int32, pin_memory=True)
    host_pr = torch.empty((V, K), dtype=torch.float32, pin_memory=True)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        g.batch(off, seeds, K=K, max_it=50, tol=1e-7, levels_out=host_lv, ppr_out=host_pr)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / a.steps, world)
    e2e = {"value": round(world * visits / (e2e_ms * 1e-3) / 1e9, 3), "unit": "G visits/s",
           "h2d_bytes_per_step": int(4 * (count + 1) + seeds.nbytes),
           "d2h_bytes_per_step": int(4 * V * (1 + K)), "ms_per_step": round(e2e_ms, 3)}
    from oracle import oracle
    extra = {}
    rp = cl = None
    if rank == 0 and (not a.no_parity or (world == 1 and not a.no_cpu_baseline)):
        rp, cl, _ = g.csr()
    if rank == 0 and not a.no_parity:
        hlv, hpr = host_lv.numpy(), host_pr.numpy()
        bfs_bad = 0
        for i in range(count):
            b, e = int(off[i]), int(off[i + 1])
            lrp = (rp[b:e + 1] - rp[b]).astype(np.uint32)
            lcl = (cl[rp[b]:rp[e]] - b).astype(np.uint32)
            ref, _ = oracle.bfs(lrp, lcl, 0)
            bfs_bad += int(np.count_nonzero(hlv[b:e] != ref))
        m = 64   # PPR of the first 64 instances (all 512 in tests/test_gpu_fullsize.py)
        pref, pit = oracle.ppr_batch(rp, cl, off[:m + 1], seeds[:m], 0.85,
                                     iters[:m].astype(np.int32), 0.0)
        b = int(off[m])
        diff = np.abs(hpr[:b].astype(np.float64) - pref[:b])
        ok = bool(np.all(diff <= 2e-5 * np.abs(pref[:b]) + 2e-7))
        extra["parity"] = {"checked": True, "vs": "oracle BFS per instance (all 512) and FP64 "
                           f"PPR-32 after the same iterations (first {m} instances)",
                           "bfs_mismatches": bfs_bad, "ppr_max_abs_err": float(diff.max()),
                           "ppr_tolerance": "|d| <= 2e-5 |ref| + 2e-7",
                           "pass": bfs_bad == 0 and ok and bool(np.all(pit == iters[:m]))}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
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
                       cpu, e2e, a.steps, clk, extra)
    g.close()
    return line


# --------------------------------------------- K-vector personalised PR --
def ppr_line(a, rank, world, local_rank):
    """32 personalised PageRank vectors on RMAT-22 (seeds uniform over vertices
    with out-degree >= 1, numpy seed 3), advanced together by olv_ppr_batch;
    a step is one solve (<= 50 iterations, tol 1e-7)."""
    import torch
    import olive_b200 as ob
    stream = torch.cuda.current_stream()
    g = ob.Graph.rmat(a.scale, 16, a.seed)
    g.set_stream(stream)
    V, E = g.V, g.E
    rp, cl, _ = g.csr()
    deg = np.diff(rp.astype(np.int64))
    K = 32
    seeds = np.random.default_rng(3).choice(np.flatnonzero(deg > 0), K,
                                            replace=False).astype(np.uint32)
    sd = torch.from_numpy(seeds.astype(np.int32)).cuda()
    out = torch.empty((V, K), dtype=torch.float32, device="cuda")

    def step():
        g.ppr(sd, 0.85, 50, 1e-7, out=out)

    for _ in range(a.warmup):
        step()
    clocks = ClockSampler(local_rank)
    clocks.start()
    barrier(world)
    ms = max_over_ranks(timed(stream, step, a.steps), world)
    clk = clocks.stop()
    st = g.last_stats
    it = st.iterations
    units = E * it                                  # edge visits (each carries K values)
    value = world * units / (ms * 1e-3) / 1e9
    peak, peak_src = peaks()
    alg = (E * (4 + 4 * K) + V * (12 * K + 8)) * it
    kern_ms = st.device_ms
    roofline = {"bound": "hbm", "achieved": round(alg / (kern_ms * 1e-3) / 1e9, 1),
                "peak": peak, "unit": "GB/s",
                "frac": round(alg / (kern_ms * 1e-3) / 1e9 / peak, 4),
                "kernel": "olv_ppr_batch solve (pull SpMM over the reverse graph, CUDA graph)",
                "algorithmic_bytes": int(alg),
                "bytes_formula": "per iteration: (4 B in-edge id + 4K B contribution row) per "
                                 "edge + (x read, x write, y write: 12K B + 8 B) per vertex",
                "peak_source": peak_src, "kernel_ms": round(kern_ms, 4)}
    traffic, traffic_src = profile_traffic("ppr", a.scale, a.seed)
    roofline.update(traffic=traffic, traffic_source=traffic_src)
    host = torch.empty((V, K), dtype=torch.float32, pin_memory=True)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        g.ppr(seeds, 0.85, 50, 1e-7, out=host)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / a.steps, world)
    e2e = {"value": round(world * units / (e2e_ms * 1e-3) / 1e9, 3), "unit": "GE/s/iter",
           "h2d_bytes_per_step": int(seeds.nbytes), "d2h_bytes_per_step": int(4 * V * K),
           "ms_per_step": round(e2e_ms, 3)}
    extra = {"K": K, "iterations": it}
    if rank == 0 and not a.no_parity:
        from oracle import oracle
        ks = [0, 31]
        ref, _ = oracle.ppr(rp, cl, seeds[ks], 0.85, it, 0.0)
        got = host.numpy()[:, ks].astype(np.float64)
        err = float(max(np.max(np.abs(got[:, j] - ref[:, j])) / np.max(ref[:, j])
                        for j in range(len(ks))))
        extra["parity"] = parity_float(err, 1e-6, f"FP64 oracle, vectors 0 and 31, the same "
                                                  f"{it} iterations (normwise per vector)")
    config = workload_config(a, V, E, None, {"K": K, "seeds": "32 distinct, out-degree >= 1",
                                             "alpha": 0.85, "max_it": 50, "tol": 1e-7})
    config["workload"] = f"ppr32-rmat{a.scale}"
    line = common_line(a, world, "GE/s/iter", value, ms, "f32",
                       "synthetic (seeded RMAT, generated on the device)", config, roofline,
                       None, e2e, a.steps * (3 * it + 4), clk, extra)
    g.close()
    return line


# ------------------------------------------------------- default extras --
def extras(a, rank, world, local_rank):
    """The other benchmarked configurations, each as a compact summary in the
    default line: msBFS-64 on RMAT-24, PageRank on RMAT-22, weighted PageRank
    forward + adjoint on RMAT-20, the ER-512 batch."""
    out = {}
    for w in ("msbfs", "pagerank", "ppr", "wpr", "batch"):
        b = copy.copy(a)
        b.workload, b.scale = w, default_scale(w)
        b.steps, b.warmup = min(a.steps, 10), 3
        b.no_cpu_baseline = True
        fn = {"wpr": wpr_line, "batch": batch_line, "ppr": ppr_line}.get(w, traversal_line)
        ln = fn(b, rank, world, local_rank) if fn is not traversal_line else \
            traversal_line(b, rank, world, local_rank, extra_keys=False)
        s = {"metric": ln["metric"], "value": ln["value"], "unit": ln["unit"],
             "ms_per_step": ln["ms_per_step"], "steps": b.steps,
             "roofline_frac": ln["roofline"]["frac"], "clocks": ln["clocks"],
             "e2e": {k: ln["e2e"][k] for k in ("value", "unit", "ms_per_step")}}
        for k in ("sequential_plain", "fwd_bwd_over_fwd", "target", "parity"):
            if k in ln:
                s[k] = ln[k]
        if "dram_frac" in ln["roofline"]:
            s["dram_frac"] = ln["roofline"]["dram_frac"]
        if w == "msbfs":
            s["target"] = ">= 10x the aggregate GTEPS of 64 sequential plain runs"
        out[w] = s
    return out


# ------------------------------------------------------------ reference --
def _ref_binary(name):
    p = os.path.join(ROOT, "oracle", "_ref", name)
    return p if os.path.exists(p) else None


def _run_ref_binary(cmd, cwd, budget_s, steps):
    """Run a reference checker binary up to `steps` times within budget_s;
    returns the loop times (ms) its own timer printed and the last stderr."""
    times, err, t0 = [], "", time.perf_counter()
    for _ in range(max(steps, 1)):
        p = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"{cmd[0]} failed: {p.stderr[-500:]}")
        err = p.stderr
        m = re.findall(r"time=?:?\s*([0-9.]+)\s*ms", err)
        if m:
            times.append(float(m[-1]))
        if time.perf_counter() - t0 > budget_s:
            break
    return times, err


def run_reference(a, rank, world):
    if rank != 0:
        return
    from oracle import oracle
    threads = oracle.max_threads()
    bound = a.ref_seconds
    vals, ms = [], []
    extra = {}
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
    deg = np.diff(rp.astype(np.int64))
    src = int(np.argmax(deg))
    kind = "port"
    if a.workload == "sssp":
        w = oracle.uint_weights_par(E, 2, 1, 255, threads)
        desc = (f"CPU restatement of SSSP.cu's frontier Bellman-Ford (edgeFilter atomicMin + "
                f"vertexFilter supersteps, oliver.h:56-113) on {threads} OpenMP threads; each "
                f"step a full solve (stopped after {max(bound, 60.0):.0f} s at most); value = "
                f"E_reached / t as for the GPU arm (sum of out-degrees of reached vertices)")
        scanned = []
        for i in range(a.warmup + a.steps):
            dist, edges, secs, rounds = oracle.sssp_frontier(rp, cl, w, src, threads,
                                                             max(bound, 60.0))
            if i >= a.warmup:
                e_reached = int(deg[dist != INF].sum())
                vals.append(e_reached / secs / 1e9)
                scanned.append(edges / secs / 1e9)
                ms.append(secs * 1e3)
        extra["edges_scanned_rate"] = {"value": round(float(np.median(scanned)), 5),
                                       "unit": "G edges scanned/s",
                                       "note": "frontier Bellman-Ford re-relaxes edges; this "
                                               "counts every scan"}
        unit, cores = "GTEPS", threads
    elif a.workload == "msbfs":
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
    elif a.workload in ("bfs", "pagerank") and _ref_binary(
            "testBFS" if a.workload == "bfs" else "testPageRank") and a.scale <= 22:
        # the reference's own serial checker, built unmodified from its sources
        name = "testBFS" if a.workload == "bfs" else "testPageRank"
        exe = _ref_binary(name)
        work = tempfile.mkdtemp(prefix="olv_ref_")
        path = os.path.join(work, "graph.txt")
        t = time.perf_counter()
        oracle.write_edge_list(path, rp, cl)
        write_s = time.perf_counter() - t
        fsize = os.path.getsize(path)
        if a.workload == "bfs":
            cmd = [exe, path, "-s", str(src)]
            _, e_reached = oracle.bfs(rp, cl, src)
            units_per_run = e_reached
        else:
            cmd = [exe, path, "-max", "50"]
        times, err = _run_ref_binary(cmd, work, 120.0, a.warmup + a.steps)
        if a.workload == "pagerank":
            it = int(re.findall(r"iterations:\s*(\d+)", err)[-1])
            sweeps = min(it + 1, 50)   # it breaks before counting the converged sweep
            units_per_run = E * sweeps
        runs = times[a.warmup:] if len(times) > a.warmup else times
        vals = [units_per_run / (t_ * 1e-3) / 1e9 for t_ in runs]
        ms = runs
        kind = "reference"
        unit, cores = ("GTEPS" if a.workload == "bfs" else "GE/s/iter"), 1
        desc = (f"oracle/_ref/{name} (the reference's serial checker compiled unmodified from "
                f"its sources), {' '.join(os.path.basename(c) for c in cmd[1:])}; its own loop "
                f"timer (file parse excluded); {len(runs)} timed runs after "
                f"{len(times) - len(runs)} warm-up; edge-list file {fsize / 1e6:.0f} MB written "
                f"in {write_s:.1f} s" + ("" if a.workload == "bfs" else
                                         "; no dangling redistribution (testPageRank.cu)"))
        shutil.rmtree(work, ignore_errors=True)
    elif a.workload == "bfs":
        desc = ("restatement of testBFS.cu:64-79 (the reference's serial queue BFS; 1 core); "
                f"each step a full traversal or stopped after {bound:.0f} s; the reference "
                f"binary is not run at this scale: its text edge list would be "
                f"{E * 19 / 1e9:.1f} GB and take minutes to parse per run")
        for i in range(a.warmup + a.steps):
            edges, secs, _ = oracle.bfs_timed(rp, cl, src, bound)
            if i >= a.warmup:
                vals.append(edges / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "GTEPS", 1
    elif a.workload == "ppr":
        K = 32
        seeds = np.random.default_rng(3).choice(np.flatnonzero(deg > 0), K,
                                                replace=False).astype(np.uint32)
        desc = ("oracle FP64 personalised PageRank, the GPU arm's 32 seeds (the reference has "
                "no PPR; 1 core); each step 2 iterations")
        for i in range(a.warmup + a.steps):
            t = time.perf_counter()
            oracle.ppr(rp, cl, seeds, 0.85, 2, 0.0)
            secs = time.perf_counter() - t
            if i >= a.warmup:
                vals.append(E * 2 / secs / 1e9)
                ms.append(secs * 1e3)
        unit, cores = "GE/s/iter", 1
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
            "dtype": "f64" if a.workload in ("pagerank", "wpr", "ppr") else "u32",
            "data": "synthetic (seeded RMAT, generated on the host)",
            "config": workload_config(a, V, E, src, {
                "weights": "lognormal(0,1) FP32, numpy seed 7", "p": "Dirichlet(1)",
                "sweeps_per_step": 2} if a.workload == "wpr" else None),
            "cpu_baseline": {"value": round(value, 5), "unit": unit, "cores": cores,
                             "kind": kind, "sample": desc},
            "e2e": {"value": round(value, 5), "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    line.update(extra)
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", a.gpus if a.gpus == 1 else 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    fn = {"wpr": wpr_line, "batch": batch_line, "ppr": ppr_line}.get(a.workload, traversal_line)
    line = fn(a, rank, world, local_rank)
    if a.workload == "sssp" and not a.no_extras:
        line.update(extras(a, rank, world, local_rank))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
