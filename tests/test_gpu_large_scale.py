"""Invariants of full-size fills, past the sizes the oracle can replay.

insertManySorted on tables with more than 2^24 buckets: the zone where the
reference's own sorted insert packs (i1 << bitsPerTag) | fp into 32 bits for
8-bit tags and so truncates bucket indices (reference CuckooFilter.cuh:159-207,
:1185-1207).  The library packs 64-bit entries (32-bit ones only where they
fit), so every key must land in one of its own two buckets.  Checked through
size-independent properties:
  * counters against the image, no lost tags, no failed insert;
  * zero false negatives over every inserted key;
  * the table's (bucket pair, tag) multiset equals the keys' (digests from the
    torch restatement of the reference's hashing, pinned to the golden vectors);
  * for a sample of keys, the oracle's candidate buckets hold the key's tag.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

import bench  # noqa: E402


@pytest.mark.parametrize("bits,bs,cap_log2", [(8, 16, 29), (32, 8, 28)])
def test_sorted_fill_past_2_24_buckets(cfb, orc, bits, bs, cap_log2):
    cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=bits, bucketSize=bs, maxEvictions=500,
                           evictionPolicy=cfb.EvictionPolicy.BFS)
    f = cfb.CuckooFilter(cfg, 1 << cap_log2)
    try:
        nb = f.getNumBuckets()
        assert nb > (1 << 24)
        n = int(0.95 * f.capacity())
        keys = torch.empty(n, dtype=torch.int64, device="cuda")
        bench.splitmix64_torch(3, 0, n, keys)
        occ = f.insertManySorted(keys)
        st = f.stats()
        assert st["failed"] == 0 and st["lost"] == 0, st
        assert occ == n == f.countOccupiedSlots(), (occ, n)
        # zero false negatives over every key
        hit = torch.empty(1 << 27, dtype=torch.bool, device="cuda")
        misses = 0
        for a in range(0, n, 1 << 27):
            m = min(1 << 27, n - a)
            f.containsManyAsync(keys[a:a + m], hit[:m])
            misses += int((~hit[:m]).sum().item())
        assert misses == 0
        # the stored multiset is exactly the keys'
        img = f.table_image()
        assert bench.table_digest(img, bits, bs, nb) == bench.key_digest(keys, bits, nb)
        # a sample through the oracle: its candidate buckets hold the tag, and the
        # torch restatement agrees with it key by key
        o = orc.OracleFilter(key_bytes=8, bits=bits, bucket_size=bs, policy=orc.POLICY_BFS, capacity=1 << cap_log2)
        idx = torch.randint(0, n, (200_000,), generator=torch.Generator().manual_seed(7))
        sample = keys[idx.cuda()].cpu().numpy().view(np.uint64)
        i1, i2, fp = o.candidates(sample)
        assert int(i1.max()) >= (1 << 24) and int(i2.max()) >= (1 << 24)
        t1, t2, tf = bench.candidates_torch(torch.from_numpy(sample.view(np.int64)), 8, bits, nb)
        assert np.array_equal(t1.numpy().view(np.uint64), i1) and np.array_equal(t2.numpy().view(np.uint64), i2)
        assert np.array_equal(tf.numpy().astype(np.uint32), fp)
        slots = img.cpu().numpy().view({8: np.uint8, 16: np.uint16, 32: np.uint32}[bits]).reshape(nb, bs)
        in1 = (slots[i1.astype(np.int64)] == fp[:, None]).any(axis=1)
        in2 = (slots[i2.astype(np.int64)] == fp[:, None]).any(axis=1)
        assert (in1 | in2).all()
    finally:
        f.close()
