"""The C++ drop-in header (include/CuckooFilter.cuh) against the reference's
behavioural test suite.

* CPU: the header compiles with a plain host compiler (no nvcc) and its static
  helpers, which run on the host through the library, return the reference's
  known answers; the nvcc-built test program (thrust overloads included) links.
* GPU: that program runs the reference's 12 unit-test scenarios
  (reference tests/test_cuckoo_filter.cu) plus the sorted insert and the error
  path, through the C ABI.
"""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "cuckoo-filter_b200", "lib")
SRC = os.path.join(ROOT, "tests", "cpp", "test_cuckoo_filter_api.cu")
OUT_DIR = os.path.join(ROOT, "tests", "cpp", "_build")
BIN = os.path.join(OUT_DIR, "test_cuckoo_filter_api")
CUDA_INC = "/usr/local/cuda/include"

HOST_PROGRAM = r"""
#include <CuckooFilter.cuh>
#include <cstdio>
int main() {
    using C16 = CuckooConfig<uint64_t, 16, 500, 256, 16, XorAltBucketPolicy, EvictionPolicy::BFS>;
    using F = CuckooFilter<C16>;
    static_assert(std::is_same_v<C16::TagType, uint16_t>, "TagType");
    static_assert(C16::evictionPolicy == EvictionPolicy::BFS, "policy");
    static_assert(CuckooConfig<uint32_t, 8>::bucketSize == 16 &&
                  CuckooConfig<uint32_t, 8>::evictionPolicy == EvictionPolicy::DFS, "defaults");
    int bad = 0;
    bad += F::hash64(1) != 0x9F29CB17A2A49995ull;
    auto [i1, i2, fp] = F::getCandidateBuckets(42, 1 << 16);
    bad += !(i1 == 17235 && i2 == 21006 && fp == 32879);
    bad += F::getAlternateBucket(i1, fp, 1 << 16) != i2;
    bad += F::calculateNumBuckets(1 << 20) != (1 << 16);
    bad += F::calculateNumBuckets(10000) != 1024;
    std::printf("%d\n", bad);
    return bad;
}
"""


def _nvcc() -> str | None:
    return shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)


def build_test_program() -> str:
    """Compile the C++ test program with nvcc (thrust overloads enabled)."""
    os.makedirs(OUT_DIR, exist_ok=True)
    if os.path.exists(BIN) and os.path.getmtime(BIN) > max(os.path.getmtime(SRC), os.path.getmtime(
            os.path.join(INC, "CuckooFilter.cuh")), os.path.getmtime(os.path.join(INC, "cuckoo_b200.h"))):
        return BIN
    cmd = [_nvcc(), "-std=c++17", "-O2", f"-I{INC}", "-gencode", "arch=compute_100a,code=sm_100a", SRC,
           f"-L{LIBDIR}", "-lcuckoo_b200", "-Xlinker", "-rpath", "-Xlinker", LIBDIR, "-o", BIN + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    os.replace(BIN + ".tmp", BIN)
    return BIN


def test_header_compiles_with_host_compiler_and_helpers_match(cfb, tmp_path):
    if not shutil.which("g++") or not os.path.isdir(CUDA_INC):
        pytest.skip("g++ or the CUDA headers are missing")
    src = tmp_path / "host.cpp"
    src.write_text(HOST_PROGRAM)
    exe = tmp_path / "host"
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", f"-I{INC}", f"-I{CUDA_INC}", str(src),
                        f"-L{LIBDIR}", "-lcuckoo_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0 and run.stdout.strip() == "0", run.stdout + run.stderr


def test_reference_suite_program_builds(cfb):
    if not _nvcc():
        pytest.skip("nvcc missing")
    assert os.path.exists(build_test_program())


@pytest.mark.gpu
def test_reference_suite_through_cpp_header(cfb):
    exe = build_test_program()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout and r.stdout.count("[  OK  ]") == 15, r.stdout
