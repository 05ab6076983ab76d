"""Build the reference's applications, unmodified, against the
source-compatible header layer in include/olive/.

    python -m olive_b200.dropin --ref <reference tree>   (or OLIVE_REFERENCE=<tree>)

BFS.cu, SSSP.cu and PageRank.cu (and testCsrGraph.cu) are symlinked from the
reference tree into olive_b200/_apps/src/, so their quoted includes
("oliver.h", "csrGraph.h", ...) resolve to include/olive/ instead of the
reference's own headers, and are compiled by nvcc for sm_100a into
olive_b200/_apps/.  Nothing is copied or edited.  Without the reference tree
the step is skipped (the built binaries travel with the repository).
"""
import argparse
import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
APPS = os.path.join(PKG, "_apps")
SRC = os.path.join(APPS, "src")
INC = os.path.join(ROOT, "include", "olive")
APP_NAMES = ["BFS", "SSSP", "PageRank", "testCsrGraph"]
# programs of this repository built the same way (tests/cpp): BFS with the
# header layer's pull opt-ins
OWN_APPS = {"BFSPullOptIn": os.path.join(ROOT, "tests", "cpp", "bfs_pull_optin.cu")}


def nvcc():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def app_path(name):
    return os.path.join(APPS, name)


def _headers():
    hs = [os.path.join(INC, h) for h in os.listdir(INC) if h.endswith(".h")]
    shared = os.path.join(ROOT, "include", "olive_b200")
    return hs + [os.path.join(shared, h) for h in os.listdir(shared) if h.endswith(".cuh")]


def _nvcc_app(src, out):
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
           "-std=c++17", "-w", "-I", INC, src, "-o", out]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"drop-in build of {os.path.basename(out)} failed:\n{' '.join(cmd)}\n"
                           f"{p.stdout}\n{p.stderr}")


def build_own_apps():
    """Build this repository's programs on the header layer (no reference needed)."""
    os.makedirs(APPS, exist_ok=True)
    built = []
    headers = _headers()
    for name, src in OWN_APPS.items():
        out = app_path(name)
        if not (os.path.exists(out) and all(os.path.getmtime(out) > os.path.getmtime(h)
                                            for h in headers + [src])):
            _nvcc_app(src, out)
        built.append(out)
    return built


def build_apps(ref=None, names=APP_NAMES):
    ref = ref or os.environ.get("OLIVE_REFERENCE")
    own = build_own_apps()
    if not ref or not os.path.exists(os.path.join(ref, "BFS.cu")):
        return own
    os.makedirs(SRC, exist_ok=True)
    built = list(own)
    headers = _headers()
    for name in names:
        src = os.path.join(SRC, name + ".cu")
        if os.path.lexists(src):
            os.unlink(src)
        os.symlink(os.path.join(ref, name + ".cu"), src)
        out = app_path(name)
        if os.path.exists(out) and all(os.path.getmtime(out) > os.path.getmtime(h)
                                       for h in headers):
            built.append(out)
            continue
        _nvcc_app(src, out)
        built.append(out)
    return built


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    a = ap.parse_args()
    for p in build_apps(a.ref):
        print(p)


if __name__ == "__main__":
    main()
