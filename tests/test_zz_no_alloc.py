"""cf_insert_sorted_noalloc: the sorted insert for callers that cannot allocate.

Some callers cannot let a library call cudaMalloc or cudaFree: a serving
process whose other streams would stall on the device-wide synchronization
those calls can cause, or a host whose device memory is already reserved by
another allocator.  cf_insert_sorted_noalloc runs the same segment-staged insert
as cf_insert_sorted on a fixed scratch area built into the library.  This file
checks, through the C ABI, that it gives the same results as the existing entry
point on the same keys: identical per-key outcomes and occupancy, and the same
stored (bucket pair, tag) multiset (which slot a tag takes inside its bucket may
differ between any two concurrent inserts, so images are compared in that
canonical form).  Covered: two calls in a row on the shared scratch, a batch of
exactly the key limit, a batch without per-key results, the key limit and the
table-size limit (clear errors, nothing inserted) and the empty batch.

The file is named to be collected last: if it fails, a run that stops at the
first failure has already run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from test_gpu_parity import dev, host_u8, image, make  # noqa: E402

CF_ERR_INVALID, CF_ERR_UNSUPPORTED = -1, -2
MAX_KEYS = 1 << 20  # CF_NOALLOC_MAX_KEYS


def canonical_entries(f, o, orc) -> np.ndarray:
    """Sorted (min(bucket, alternate bucket), tag) of every stored tag."""
    slots = image(f).view(np.uint16).reshape(o.nb, o.bucket_size)
    b, s = np.nonzero(slots)
    tags = slots[b, s].astype(np.uint64)
    alt = orc.alt_vectorized(16, o.nb)(b.astype(np.uint64), tags)
    lo = np.minimum(b.astype(np.uint64), alt)
    return np.sort(lo * np.uint64(1 << 16) + tags)


def insert_sorted(L, f, keys, out, noalloc: bool) -> int:
    occ = C.c_uint64()
    fn = L.cf_insert_sorted_noalloc if noalloc else L.cf_insert_sorted
    st = fn(f.handle, keys.data_ptr(), keys.numel(), None if out is None else out.data_ptr(), None, C.byref(occ))
    assert st == 0, L.cf_last_error().decode()
    return int(occ.value)


def same_fill(cfb, orc, capacity, batches, with_out=True):
    """Two filters filled batch by batch, one through cf_insert_sorted and one
    through cf_insert_sorted_noalloc; asserts equal results after every batch."""
    L = cfb.library()
    a, o = make(cfb, orc, 8, 16, 16, 0, 500, capacity)
    b, _ = make(cfb, orc, 8, 16, 16, 0, 500, capacity)
    try:
        for call, keys_h in enumerate(batches):
            keys = dev(keys_h)
            out_a = out_b = None
            if with_out:
                out_a = torch.zeros(len(keys_h), dtype=torch.bool, device="cuda")
                out_b = torch.ones(len(keys_h), dtype=torch.bool, device="cuda")  # must be overwritten
            occ_a = insert_sorted(L, a, keys, out_a, noalloc=False)
            occ_b = insert_sorted(L, b, keys, out_b, noalloc=True)
            if with_out:
                assert torch.equal(out_a, out_b), f"call {call}: per-key results differ"
            assert occ_a == occ_b == a.countOccupiedSlots() == b.countOccupiedSlots(), (call, occ_a, occ_b)
            assert a.stats()["failed"] == b.stats()["failed"] == 0
            assert b.stats()["lost"] == 0
            assert np.array_equal(canonical_entries(a, o, orc), canonical_entries(b, o, orc)), call
            assert host_u8(b.containsMany(keys)).all(), "false negative"
    finally:
        a.close()
        b.close()


def test_noalloc_two_calls_in_a_row_match_sorted_insert(cfb, orc):
    assert cfb.library().cf_noalloc_scratch_bytes() >= 8 * MAX_KEYS
    n = int(0.45 * (1 << 20))
    # two calls in a row on the same scratch: 0.45 then 0.9 load
    same_fill(cfb, orc, 1 << 20, [orc.splitmix64(11, n), orc.splitmix64(12, n)])


def test_noalloc_batch_of_exactly_the_key_limit(cfb, orc):
    # 2^20 buckets: the segment starts and the radix grid at their sizes for this table
    same_fill(cfb, orc, 1 << 24, [orc.splitmix64(21, MAX_KEYS), orc.splitmix64(22, MAX_KEYS)])


def test_noalloc_without_per_key_results(cfb, orc):
    n = int(0.5 * (1 << 20))
    same_fill(cfb, orc, 1 << 20, [orc.splitmix64(31, n), orc.splitmix64(32, n // 2)], with_out=False)


def test_noalloc_limits_and_empty_batch(cfb, orc):
    L = cfb.library()
    b, _ = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 20)
    try:
        b.insertManySorted(dev(orc.splitmix64(41, 1000)))
        before = b.occupiedSlots()
        occ = C.c_uint64()
        # beyond the fixed scratch: a clear error, nothing inserted
        big = torch.zeros(MAX_KEYS + 1, dtype=torch.int64, device="cuda")
        st = L.cf_insert_sorted_noalloc(b.handle, big.data_ptr(), MAX_KEYS + 1, None, None, C.byref(occ))
        assert st == CF_ERR_INVALID and b"limit" in L.cf_last_error()
        assert b.occupiedSlots() == before
        # an empty batch is a no-op
        assert L.cf_insert_sorted_noalloc(b.handle, None, 0, None, None, C.byref(occ)) == 0
        assert occ.value == before
    finally:
        b.close()
    # a table of 2^18 + 1 segments of 64 KiB (16 GiB + 64 KiB; the Offset
    # policy allows a bucket count that is not a power of two): refused
    # before anything runs
    cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=16, bucketSize=16, AltBucketPolicy="OffsetAltBucketPolicy",
                           evictionPolicy=cfb.EvictionPolicy.BFS)
    big_table = cfb.CuckooFilter(cfg, (1 << 33) + 16 * 2048)
    try:
        assert big_table.getNumBuckets() == (1 << 29) + 2048
        keys = dev(orc.splitmix64(42, 64))
        st = L.cf_insert_sorted_noalloc(big_table.handle, keys.data_ptr(), 64, None, None, C.byref(occ))
        assert st == CF_ERR_UNSUPPORTED and b"segment" in L.cf_last_error()
        assert big_table.occupiedSlots() == 0
    finally:
        big_table.close()
