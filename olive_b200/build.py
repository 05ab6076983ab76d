"""Build libolive_b200.so in-tree for sm_100a.

    python -m olive_b200.build [--jobs N] [--force]

Each olive_b200/csrc/*.cu is compiled by nvcc into olive_b200/_build/*.o and
linked with the static CUDA runtime into olive_b200/libolive_b200.so, so the
library loads on a machine without a matching libcudart.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libolive_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O2", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
]


def nvcc():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(
        os.path.join(ROOT, "include", "*.h")) + glob.glob(
        os.path.join(ROOT, "include", "olive_b200", "*.cuh"))


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def compile_one(src, force=False, extra=()):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if not force and not _stale(obj, src, _headers()):
        return obj, None
    cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    return obj, p.stderr


def build(jobs=None, force=False, verbose=False, extra=()):
    # OLV_NVCC_EXTRA: extra nvcc flags (e.g. -DOLV_ITEMS=8 to change the edges each
    # thread of the advance keeps in flight); a changed value forces a rebuild
    env_extra = os.environ.get("OLV_NVCC_EXTRA", "").split()
    stamp = os.path.join(BUILD, "flags.txt")
    os.makedirs(BUILD, exist_ok=True)
    if env_extra or os.path.exists(stamp):
        old = open(stamp).read() if os.path.exists(stamp) else ""
        if old != " ".join(env_extra):
            force = True
            with open(stamp, "w") as f:
                f.write(" ".join(env_extra))
    extra = list(extra) + env_extra
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: compile_one(s, force, extra), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    if force or not os.path.exists(LIB) or any(
            os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/smem usage")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(a.jobs, a.force or a.ptxas_v, verbose=a.ptxas_v, extra=extra))


if __name__ == "__main__":
    main()
