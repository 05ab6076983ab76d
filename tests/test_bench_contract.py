"""CPU checks of bench.py's reference arm: one JSON line per run with the
contract's keys, for every workload, and silence on ranks other than 0."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
        "cpu_baseline", "e2e"}


def _run(args, env=None):
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args,
                       capture_output=True, text=True, timeout=300, cwd=ROOT,
                       env=dict(os.environ, **(env or {})))
    assert p.returncode == 0, p.stderr[-2000:]
    return [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]


@pytest.mark.parametrize("workload,scale", [("sssp", 10), ("bfs", 10), ("pagerank", 10),
                                            ("msbfs", 10), ("wpr", 10), ("batch", 0),
                                            ("ppr", 10)])
def test_reference_arm_line(workload, scale):
    lines = _run(["--impl", "reference", "--workload", workload, "--scale", str(scale),
                  "--steps", "2", "--warmup", "1", "--ref-seconds", "0.5"])
    assert len(lines) == 1
    d = lines[0]
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith(workload)
    if workload == "batch":   # the GPU arm's 512 ER instances, 8 edges per vertex
        assert d["config"]["instances"] == 512 and d["unit"] == "G visits/s"
        assert d["config"]["E"] == 8 * d["config"]["V"]


def test_reference_arm_other_ranks_are_silent():
    lines = _run(["--impl", "reference", "--scale", "10", "--steps", "1", "--warmup", "0"],
                 env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert lines == []
