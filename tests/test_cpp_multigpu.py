"""The C++ drop-in include/CuckooFilterMultiGPU.cuh (the reference's
CuckooFilterMultiGPU<Config>): it builds with nvcc against the library (CPU),
and its test program passes on a GPU with every shard on that GPU."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "cuckoo-filter_b200", "lib")
SRC = os.path.join(ROOT, "tests", "cpp", "test_multigpu_api.cu")
OUT_DIR = os.path.join(ROOT, "tests", "cpp", "_build")
BIN = os.path.join(OUT_DIR, "test_multigpu_api")


def _nvcc() -> str | None:
    return shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)


def build_program() -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [SRC] + [os.path.join(INC, h) for h in ("CuckooFilter.cuh", "CuckooFilterMultiGPU.cuh", "cuckoo_b200.h")]
    if os.path.exists(BIN) and os.path.getmtime(BIN) > max(os.path.getmtime(d) for d in deps):
        return BIN
    cmd = [_nvcc(), "-std=c++17", "-O2", f"-I{INC}", "-gencode", "arch=compute_100a,code=sm_100a", SRC,
           f"-L{LIBDIR}", "-lcuckoo_b200", "-Xlinker", "-rpath", "-Xlinker", LIBDIR, "-o", BIN + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    os.replace(BIN + ".tmp", BIN)
    return BIN


def test_multigpu_program_builds(cfb):
    if not _nvcc():
        pytest.skip("nvcc missing")
    assert os.path.exists(build_program())


@pytest.mark.gpu
def test_multigpu_header_on_one_gpu(cfb):
    exe = build_program()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout and r.stdout.count("[  OK  ]") == 5, r.stdout
