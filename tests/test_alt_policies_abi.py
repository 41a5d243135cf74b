"""The library's host-side policy helpers (cf_hash_candidates, cf_alt_buckets,
cf_num_buckets_for_policy) for the AddSub and Offset policies, against the
reference's own policy code compiled from its headers.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

NAMES = {0: "XorAltBucketPolicy", 1: "AddSubAltBucketPolicy", 2: "OffsetAltBucketPolicy"}


@pytest.mark.parametrize("alt", [1, 2])
@pytest.mark.parametrize("kb,bits", [(8, 16), (4, 16), (8, 8), (8, 32)])
def test_host_candidates_and_alternates_match_reference(cfb, orc, alt, kb, bits):
    if orc.ref_host() is None:
        pytest.skip("oracle/_ref/libref_host.so not built")
    nb = 250_006
    cfg = cfb.CuckooConfig(T="uint64" if kb == 8 else "uint32", bitsPerTag=bits, AltBucketPolicy=NAMES[alt])
    keys = orc.splitmix64(3 + alt + bits, 10_000)
    if kb == 4:
        keys = keys.astype(np.uint32)
    got = cfb.CuckooFilter.getCandidateBuckets(cfg, keys, nb)
    want = orc.ref_candidates_policy(alt, kb, bits, nb, keys)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    i1, i2, fp = got
    alt_b, new_tag = orc.ref_alt_policy(alt, bits, nb, i1, fp)
    out = np.empty(len(i1), np.uint64)
    import ctypes as C

    c = cfg.to_c()
    assert cfb.library().cf_alt_buckets(C.byref(c), nb, i1.ctypes.data, fp.ctypes.data, len(i1), out.ctypes.data) == 0
    assert np.array_equal(out, alt_b) and np.array_equal(out, i2)


@pytest.mark.parametrize("alt", [0, 1, 2])
def test_bucket_counts(cfb, orc, alt):
    for cap in (1, 17, 4048, 1 << 20, 3_000_001):
        assert cfb.CuckooFilter.calculateNumBuckets(cap, 16, NAMES[alt]) == orc.num_buckets(cap, 16, alt)


def test_addsub_needs_an_even_bucket_count(cfb):
    import ctypes as C

    c = cfb.CuckooConfig(T="uint64", bitsPerTag=16, AltBucketPolicy="AddSubAltBucketPolicy").to_c()
    b = np.zeros(1, np.uint64)
    t = np.ones(1, np.uint32)
    out = np.zeros(1, np.uint64)
    assert cfb.library().cf_alt_buckets(C.byref(c), 1001, b.ctypes.data, t.ctypes.data, 1, out.ctypes.data) != 0
