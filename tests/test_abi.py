"""C-ABI library checks that need no GPU.

* ``libcuckoo_b200.so`` loads and exports every function ``include/*.h`` declares;
* host-side hashing exported by the library (``cf_hash_candidates``, the same
  constexpr code the kernels use) equals the reference's golden vectors;
* argument validation and status codes.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions() -> set[str]:
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(cf_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(cfb):
    L = cfb.library()
    names = declared_functions()
    assert len(names) >= 25, names
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version(cfb):
    assert cfb.library().cf_abi_version() == 1


def test_status_strings(cfb):
    L = cfb.library()
    for code, name in cfb.STATUS.items():
        assert L.cf_status_string(code).decode() == name


@pytest.mark.parametrize("kb", [8, 4])
def test_host_hashing_matches_reference_golden(cfb, golden, kb):
    i = 0
    checked = 0
    while f"c{i}_meta" in golden:
        ckb, bits, bs, cap, nb = (int(x) for x in golden[f"c{i}_meta"])
        if ckb == kb:
            cfg = cfb.CuckooConfig(T="uint64" if kb == 8 else "uint32", bitsPerTag=bits, bucketSize=bs)
            i1, i2, fp = cfb.CuckooFilter.getCandidateBuckets(cfg, golden[f"c{i}_keys"], nb)
            assert np.array_equal(i1, golden[f"c{i}_i1"]), i
            assert np.array_equal(i2, golden[f"c{i}_i2"]), i
            assert np.array_equal(fp, golden[f"c{i}_fp"]), i
            checked += 1
        i += 1
    assert checked >= 3


def test_hash64_and_alt_buckets_match_reference_golden(cfb, golden):
    """cf_hash64 (static hash64) and cf_alt_buckets (static getAlternateBucket)
    against the reference's own xxhash64 outputs and candidate pairs."""
    L = cfb.library()
    i = 0
    while f"c{i}_meta" in golden:
        kb, bits, bs, cap, nb = (int(x) for x in golden[f"c{i}_meta"])
        keys = np.ascontiguousarray(golden[f"c{i}_keys"])
        h = np.empty(len(keys), np.uint64)
        assert L.cf_hash64(kb, keys.ctypes.data, len(keys), h.ctypes.data) == 0
        assert np.array_equal(h, golden[f"c{i}_hash"]), i
        cfg = _cfg(cfb, T="uint64" if kb == 8 else "uint32", bitsPerTag=bits, bucketSize=bs)
        i1 = np.ascontiguousarray(golden[f"c{i}_i1"])
        fp = np.ascontiguousarray(golden[f"c{i}_fp"])
        out = np.empty(len(keys), np.uint64)
        assert L.cf_alt_buckets(C.byref(cfg), nb, i1.ctypes.data, fp.ctypes.data, len(keys), out.ctypes.data) == 0
        assert np.array_equal(out, golden[f"c{i}_i2"]), i
        i += 1
    for bits in (8, 16, 32):
        tags = np.ascontiguousarray(golden[f"tag{bits}"].astype({8: np.uint8, 16: np.uint16, 32: np.uint32}[bits]))
        h = np.empty(len(tags), np.uint64)
        assert L.cf_hash64(bits // 8, tags.ctypes.data, len(tags), h.ctypes.data) == 0
        assert np.array_equal(h, golden[f"taghash{bits}"]), bits
    assert L.cf_hash64(3, None, 0, None) == -1


def test_num_buckets_matches_reference(cfb, golden):
    for cap, bs, nb in golden["num_buckets"]:
        assert cfb.CuckooFilter.calculateNumBuckets(int(cap), int(bs)) == int(nb)


def _cfg(cfb, **kw):
    base = dict(T="uint64", bitsPerTag=16)
    base.update(kw)
    return cfb.CuckooConfig(**base).to_c()


def test_config_support_matrix(cfb):
    L = cfb.library()
    for bits, sizes in ((8, (8, 16, 32, 64)), (16, (4, 8, 16, 32, 64, 128)), (32, (2, 4, 8, 16))):
        for bs in sizes:
            for t in ("uint64", "uint32"):
                assert L.cf_config_supported(C.byref(_cfg(cfb, T=t, bitsPerTag=bits, bucketSize=bs)))
    assert not L.cf_config_supported(C.byref(_cfg(cfb, bitsPerTag=8, bucketSize=4)))
    assert not L.cf_config_supported(C.byref(_cfg(cfb, bitsPerTag=16, bucketSize=256)))
    assert not L.cf_config_supported(C.byref(_cfg(cfb, bitsPerTag=32, bucketSize=32)))


@pytest.mark.parametrize("kw,status", [
    (dict(bitsPerTag=12), -1),
    (dict(bucketSize=12), -1),
    (dict(maxEvictions=0), -1),
    (dict(maxEvictions=513), -1),
    (dict(blockSize=100), -1),
    (dict(bitsPerTag=16, bucketSize=256), -2),
])
def test_create_rejects_bad_configs(cfb, kw, status):
    L = cfb.library()
    h = C.c_void_p()
    rc = L.cf_create(C.byref(_cfg(cfb, **kw)), 1 << 10, C.byref(h))
    assert rc == status, L.cf_last_error()
    assert not h.value
    assert L.cf_last_error().decode()


def test_null_arguments(cfb):
    L = cfb.library()
    assert L.cf_destroy(None) == 0
    assert L.cf_contains(None, None, 0, None, None) == -1
    assert L.cf_create(C.byref(_cfg(cfb)), 1024, None) == -1
    assert L.cf_hash_candidates(None, 16, None, 0, None, None, None) == -1
    assert L.cf_hash_candidates(C.byref(_cfg(cfb)), 12, None, 0, None, None, None) == -1


def test_create_without_gpu_fails_cleanly(cfb):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = cfb.library()
    h = C.c_void_p()
    rc = L.cf_create(C.byref(_cfg(cfb)), 1 << 10, C.byref(h))
    assert rc in (-6, -3), rc
    assert not h.value


def test_python_config_mirror(cfb):
    c = cfb.CuckooConfig(T="uint64_t", bitsPerTag=16)
    assert (c.maxEvictions, c.blockSize, c.bucketSize, c.evictionPolicy) == (500, 256, 16, cfb.EvictionPolicy.DFS)
    assert c.TagType == "uint16_t" and c.key_bytes == 8
    assert cfb.CuckooConfig(T="uint64", bitsPerTag=16, AltBucketPolicy="AddSubAltBucketPolicy").to_c().alt_policy == 1
    assert cfb.CuckooConfig(T="uint64", bitsPerTag=16, AltBucketPolicy="OffsetAltBucketPolicy").to_c().alt_policy == 2
    with pytest.raises(cfb.CuckooError):
        cfb.CuckooConfig(T="uint64", bitsPerTag=16, AltBucketPolicy="ModuloAltBucketPolicy").to_c()


def test_python_option_constants_match_the_header(cfb):
    """Every CF_OPT_* and CF_STAGING_* value of include/cuckoo_b200.h has a
    Python constant of the same name (without the CF_ prefix) and value."""
    text = open(os.path.join(ROOT, "include", "cuckoo_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    found = dict((m.group(1), int(m.group(2))) for m in re.finditer(r"\bCF_((?:OPT|STAGING)_\w+)\s*=\s*(\d+)", text))
    assert "OPT_PROBE_WIDTH" in found and "STAGING_REGION" in found
    for name, value in found.items():
        assert getattr(cfb, name) == value, name
