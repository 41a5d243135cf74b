"""cf_insert_sorted_noalloc: the sorted insert for callers that cannot allocate.

Some callers cannot let a library call cudaMalloc or cudaFree: a serving
process whose other streams would stall on the implicit device
synchronization, a stream under CUDA-graph capture, a host whose device memory
is already reserved by another allocator.  cf_insert_sorted_noalloc runs the
same segment-staged insert as cf_insert_sorted on a fixed scratch area built
into the library.  This file checks, through the C ABI, that two calls in a row
give the same results as the existing entry point on the same keys: identical
per-key outcomes and occupancy, and the same stored (bucket pair, tag)
multiset (which slot a tag takes inside its bucket may differ between any two
concurrent inserts, so images are compared in that canonical form).  It also
checks the size limit and the empty batch.

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
    st = fn(f.handle, keys.data_ptr(), keys.numel(), out.data_ptr(), None, C.byref(occ))
    assert st == 0, L.cf_last_error().decode()
    return int(occ.value)


def test_noalloc_sorted_insert_matches_sorted_insert(cfb, orc):
    L = cfb.library()
    assert L.cf_noalloc_scratch_bytes() >= 8 * (1 << 20)
    a, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 20)
    b, _ = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 20)
    limit = 1 << 20
    # two calls in a row on the same scratch: 0.45 then 0.9 load
    for call, seed in enumerate((11, 12)):
        keys_h = orc.splitmix64(seed, int(0.45 * a.capacity()))
        keys = dev(keys_h)
        out_a = torch.zeros(len(keys_h), dtype=torch.bool, device="cuda")
        out_b = torch.ones(len(keys_h), dtype=torch.bool, device="cuda")  # must be overwritten
        occ_a = insert_sorted(L, a, keys, out_a, noalloc=False)
        occ_b = insert_sorted(L, b, keys, out_b, noalloc=True)
        assert torch.equal(out_a, out_b), f"call {call}: per-key results differ"
        assert occ_a == occ_b == a.countOccupiedSlots() == b.countOccupiedSlots(), (call, occ_a, occ_b)
        assert a.stats()["failed"] == b.stats()["failed"] == 0
        assert np.array_equal(canonical_entries(a, o, orc), canonical_entries(b, o, orc)), call
        assert host_u8(b.containsMany(keys)).all(), "false negative"
    # beyond the fixed scratch: a clear error, nothing inserted
    big = torch.zeros(limit + 1, dtype=torch.int64, device="cuda")
    before = b.occupiedSlots()
    occ = C.c_uint64()
    st = L.cf_insert_sorted_noalloc(b.handle, big.data_ptr(), limit + 1, None, None, C.byref(occ))
    assert st == -1 and b"limit" in L.cf_last_error()
    assert b.occupiedSlots() == before
    # an empty batch is a no-op
    assert L.cf_insert_sorted_noalloc(b.handle, None, 0, None, None, C.byref(occ)) == 0
    assert occ.value == before
