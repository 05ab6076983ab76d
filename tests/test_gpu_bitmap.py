"""The source-compatible Bitmap (include/olive/bitmap.h, the reference's
bitmap.h:44-199): a small CUDA program built against the header layer sets and
clears bits from device threads and checks get/count and the &, |, ^
operators on the host."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "bitmap_check.cu")


def _build(out):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
           "-I", os.path.join(ROOT, "include", "olive"), SRC, "-o", out]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]


def test_bitmap_header_compiles_for_sm100a(tmp_path):
    _build(str(tmp_path / "bitmap_check"))


@pytest.mark.gpu
def test_bitmap_on_gpu(tmp_path):
    exe = str(tmp_path / "bitmap_check")
    _build(exe)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "bitmap ok" in p.stdout
