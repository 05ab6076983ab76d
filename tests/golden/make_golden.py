"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a container where the reference tree exists:

    python tests/golden/make_golden.py --ref <reference tree>   (or OLIVE_REFERENCE=<tree>)

It builds the reference's own serial checkers (oracle/Makefile -> oracle/_ref)
and records, for every graph file in the reference's data/ directory:
  * the CSR exactly as the reference loader builds it (csrGraph.h:106-171),
    and the CSR with tuples stably sorted by source;
  * BFS levels from testBFS (testBFS.cu:42-87) for every source (all sources
    of graphs up to 100 vertices, 0 plus 63 evenly spaced ones otherwise);
  * PageRank from testPageRank (testPageRank.cu:41-115): the printed ranks
    ("%f") and iteration count, default -max and -max 50.
It also writes the 128x128 grid and two small RMAT graphs as edge lists, runs
the same checkers on them, and stores levels, ranks and a CSR checksum.
"""
import argparse
import glob
import hashlib
import os
import re
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def csr_digest(rowptr, col):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rowptr, np.uint32).tobytes())
    h.update(np.ascontiguousarray(col, np.uint32).tobytes())
    return h.hexdigest()


def pr_iters(stderr):
    m = re.search(r"iterations:\s*(\d+)", stderr)
    return int(m.group(1))


def record(path, name, work, srcs_all_limit=100):
    rowptr, col, w = oracle.load_edge_list_ref(path)
    V = len(rowptr) - 1
    if V <= srcs_all_limit:
        srcs = np.arange(V, dtype=np.int64)
    else:
        srcs = np.unique(np.concatenate([[0], np.linspace(0, V - 1, 63).astype(np.int64)]))
    levels = np.stack([oracle.run_ref_bfs(path, int(s), work)[0] for s in srcs])
    pr, err = oracle.run_ref_pagerank(path, work)
    pr50, err50 = oracle.run_ref_pagerank(path, work, 50)
    srow, scol, sw = oracle.load_edge_list_sorted(path)
    out = dict(rowptr=rowptr, col=col, sorted_rowptr=srow, sorted_col=scol,
               bfs_sources=srcs.astype(np.uint32), bfs_levels=levels.astype(np.int32),
               pr_ranks=pr, pr_iterations=np.int64(pr_iters(err)),
               pr50_ranks=pr50, pr50_iterations=np.int64(pr_iters(err50)))
    if w is not None:
        out["weights"] = w
        out["sorted_weights"] = sw
    np.savez_compressed(os.path.join(OUT, f"fixture_{name}.npz"), **out)
    print(f"{name}: V={V} E={len(col)} sources={len(srcs)} pr_it={out['pr_iterations']}")


def record_generated(name, rowptr, col, srcs, work, pr=True):
    path = os.path.join(work, name + ".txt")
    oracle.write_edge_list(path, rowptr, col)
    levels = np.stack([oracle.run_ref_bfs(path, int(s), work)[0] for s in srcs])
    out = dict(digest=np.array(csr_digest(rowptr, col)), V=np.int64(len(rowptr) - 1),
               E=np.int64(len(col)), bfs_sources=np.asarray(srcs, np.uint32),
               bfs_levels=levels.astype(np.int32))
    if pr:
        r50, err50 = oracle.run_ref_pagerank(path, work, 50)
        out["pr50_ranks"] = r50
        out["pr50_iterations"] = np.int64(pr_iters(err50))
    np.savez_compressed(os.path.join(OUT, f"gen_{name}.npz"), **out)
    print(f"{name}: V={len(rowptr) - 1} E={len(col)} sources={len(srcs)}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("OLIVE_REFERENCE"),
                    help="the reference source tree (or set OLIVE_REFERENCE)")
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the reference tree with --ref or OLIVE_REFERENCE")
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={a.ref}"],
                   check=True)
    with tempfile.TemporaryDirectory() as work:
        for path in sorted(glob.glob(os.path.join(a.ref, "data", "*"))):
            record(path, os.path.basename(path), work)
        rp, cl = oracle.grid_csr(128, 128)
        record_generated("grid_128x128", rp, cl, [0, 8256, 16383], work)
        for scale in (10, 12):
            rp, cl = oracle.rmat_csr(scale, 16, 1)
            deg = np.diff(rp.astype(np.int64))
            hub = int(np.argmax(deg))
            rng = np.random.default_rng(scale)
            others = rng.choice(np.flatnonzero(deg > 0), 3, replace=False)
            record_generated(f"rmat{scale}_ef16_s1", rp, cl, [hub, *others.tolist()], work)


if __name__ == "__main__":
    main()
