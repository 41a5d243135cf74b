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


HOST_PROGRAM = r"""
#include <CuckooFilterMultiGPU.cuh>
#include <cstdio>
#include <vector>
using C = CuckooConfig<uint64_t, 16, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS>;
int main(int argc, char**) {
    if (argc > 5) {  // every member instantiated; nothing runs without a GPU
        CuckooFilterMultiGPU<C> f(2, 1 << 20);
        std::vector<uint64_t> k(10);
        std::vector<bool> o;
        f.insertMany(k);
        f.containsMany(k, o);
        f.deleteMany(k, o);
        f.deleteMany(k);
        std::printf("%f %zu %zu %zu\n", f.loadFactor(), f.totalOccupiedSlots(), f.totalCapacity(), f.sizeInBytes());
        f.clear();
        f.synchronizeAllGPUs();
    }
    std::printf("0\n");
    return 0;
}
"""


def test_multigpu_header_compiles_with_host_compiler(cfb, tmp_path):
    cuda = "/usr/local/cuda"
    if not shutil.which("g++") or not os.path.isdir(os.path.join(cuda, "include")):
        pytest.skip("g++ or the CUDA headers are missing")
    src = tmp_path / "host.cpp"
    src.write_text(HOST_PROGRAM)
    exe = tmp_path / "host"
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", f"-I{INC}", f"-I{cuda}/include", str(src),
                        f"-L{LIBDIR}", "-lcuckoo_b200", f"-Wl,-rpath,{LIBDIR}", f"-L{cuda}/lib64", "-lcudart",
                        f"-Wl,-rpath,{cuda}/lib64", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0 and run.stdout.strip() == "0", run.stdout + run.stderr
