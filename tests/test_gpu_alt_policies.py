"""AddSub and Offset alternate-bucket policies on the GPU (reference
include/bucket_policies.cuh:95-350, used by the filter at
CuckooFilter.cuh:1033-1059, :1091-1094, :1109-1112 and in its evictions).

Exact checks against the oracle: one-key-per-call insert images (evictions,
failed chains and their undo included), lookups on identical images, one-key
deletes.  The oracle's policy code is pinned to the reference's own kernels
built with these policies.  Bulk batches are checked through invariants (the
Offset policy's choice bit is set exactly on tags in their alternate bucket),
on the random, segment- and region-staged paths and in filter sets.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from test_gpu_parity import dev, host_u8, image  # noqa: E402

NAMES = {1: "AddSubAltBucketPolicy", 2: "OffsetAltBucketPolicy"}


def make(cfb, orc, alt, kb=8, policy=1, max_ev=500, cap=1 << 12):
    cfg = cfb.CuckooConfig(T="uint64" if kb == 8 else "uint32", bitsPerTag=16, bucketSize=16, maxEvictions=max_ev,
                           evictionPolicy=cfb.EvictionPolicy(policy), AltBucketPolicy=NAMES[alt])
    f = cfb.CuckooFilter(cfg, cap)
    o = orc.OracleFilter(key_bytes=kb, bits=16, bucket_size=16, policy=policy, max_evictions=max_ev, capacity=cap,
                         mode=orc.MODE_CONSERVING, alt_policy=alt)
    assert f.getNumBuckets() == o.nb == cfb.CuckooFilter.calculateNumBuckets(cap, 16, NAMES[alt])
    return f, o


SEQ = [
    # alt, key_bytes, eviction policy, max_ev, capacity (not a power of two: 16 * 250 + 16 * 3), fill
    (1, 8, 0, 500, 4048, 0.97),
    (1, 8, 1, 500, 4048, 0.97),
    (2, 8, 0, 500, 4048, 0.97),
    (2, 8, 1, 500, 4048, 0.97),
    (2, 4, 0, 500, 4048, 0.97),
    (1, 4, 1, 500, 4048, 0.97),
    (2, 8, 1, 16, 4048, 1.00),
    (1, 8, 1, 16, 4048, 1.00),
    (2, 8, 0, 16, 4000, 1.00),
]


@pytest.mark.parametrize("alt,kb,policy,max_ev,cap,fill", SEQ)
def test_sequential_image_bit_exact(cfb, orc, alt, kb, policy, max_ev, cap, fill):
    f, o = make(cfb, orc, alt, kb, policy, max_ev, cap)
    keys = orc.splitmix64(500 + alt * 10 + policy, int(fill * f.capacity()))
    if kb == 4:
        keys = keys.astype(np.uint32)
    d = dev(keys)
    out = torch.empty(1, dtype=torch.bool, device="cuda")
    got = np.empty(len(keys), np.uint8)
    for i in range(len(keys)):
        f.insertMany(d[i:i + 1], d_output=out)
        got[i] = int(out.item())
    n_ok, want = o.insert(keys, out=True)
    assert np.array_equal(got, want), f"first differing key {int(np.argmax(got != want))}"
    assert np.array_equal(image(f), o.table)
    st = f.stats()
    assert st["occupied"] == n_ok == f.countOccupiedSlots() and st["lost"] == 0
    if fill >= 1.0:
        assert st["failed"] > 0, "case meant to exercise failed chains"


@pytest.mark.parametrize("cfg_key,cap", [((2, 0, 500), 4048), ((2, 1, 500), 4048), ((1, 0, 500), 4048),
                                         ((1, 1, 500), 4048), ((2, 1, 16), 4048), ((1, 1, 16), 4048)])
def test_reference_kernels_with_policy_match_oracle(cfb, orc, cfg_key, cap):
    """The reference's own kernels with the policy, one key per launch, against
    the oracle's reference mode up to the first failed chain."""
    if orc.ref_gpu() is None:
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    alt, policy, max_ev = cfg_key
    ref = orc.RefGpuFilter(8, 16, 16, policy, max_ev, cap, alt_policy=alt)
    scratch = None
    try:
        o = orc.OracleFilter(key_bytes=8, bits=16, bucket_size=16, policy=policy, max_evictions=max_ev,
                             capacity=cap, mode=orc.MODE_REFERENCE, alt_policy=alt)
        assert ref.num_buckets() == o.nb
        cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=16, bucketSize=16, AltBucketPolicy=NAMES[alt])
        scratch = cfb.CuckooFilter(cfg, cap)
        ptr, nbytes = ref.table()
        keys = orc.splitmix64(800 + alt * 10 + policy, int(0.98 * o.nb * 16))
        d = dev(keys)
        prev = 0
        for i in range(len(keys)):
            occ = ref.insert(d[i:i + 1].data_ptr(), 1)
            ok = occ - prev
            prev = occ
            want = o.insert(keys[i:i + 1])
            assert ok == want, i
            if want == 0 or i == len(keys) - 1 or i % 500 == 0:
                scratch.load_table(ptr, nbytes)
                assert np.array_equal(image(scratch), o.table), f"image differs after key {i}"
            if want == 0:
                break
    finally:
        ref.close()
        if scratch is not None:
            scratch.close()


@pytest.mark.parametrize("alt", [1, 2])
def test_contains_and_delete_on_identical_image(cfb, orc, alt):
    f, o = make(cfb, orc, alt, cap=50_000)
    keys = orc.splitmix64(61 + alt, int(0.95 * f.capacity()))
    o.insert(keys)
    f.load_table(torch.from_numpy(o.table).cuda())
    neg = orc.splitmix64(62 + alt, 100_000)
    q = np.concatenate([keys, neg])
    assert np.array_equal(host_u8(f.containsMany(dev(q))), o.contains(q))
    dels = np.concatenate([keys[::3], orc.splitmix64(63, 200), keys[:50]])
    d = dev(dels)
    out = torch.empty(1, dtype=torch.bool, device="cuda")
    got = np.empty(len(dels), np.uint8)
    for i in range(len(dels)):
        f.deleteMany(d[i:i + 1], out)
        got[i] = int(out.item())
    _, want = o.delete(dels)
    assert np.array_equal(got, want)
    assert np.array_equal(image(f), o.table)


@pytest.mark.parametrize("sorted_", [False, True])
@pytest.mark.parametrize("alt,policy", [(1, 0), (1, 1), (2, 0), (2, 1)])
def test_bulk_invariants(cfb, orc, alt, policy, sorted_):
    f, o = make(cfb, orc, alt, policy=policy, cap=1_000_000)
    keys = orc.splitmix64(1, int(0.95 * f.capacity()))
    d = dev(keys)
    ok_t = torch.empty(len(keys), dtype=torch.bool, device="cuda")
    occ = f.insertManySorted(d, d_output=ok_t) if sorted_ else f.insertMany(d, d_output=ok_t)
    ok = host_u8(ok_t).astype(bool)
    st = f.stats()
    assert occ == ok.sum() == st["occupied"] == f.countOccupiedSlots() and st["lost"] == 0
    assert st["failed"] == len(keys) - ok.sum() and st["failed"] <= len(keys) // 1000
    assert host_u8(f.containsMany(d[torch.from_numpy(ok).cuda()])).all(), "false negative"
    slots = image(f).view(np.uint16).reshape(o.nb, 16)
    stored = keys[ok]
    i1, i2, fp = o.candidates(stored)
    errs = orc.check_invariants(slots, o.alt_map(), i1, i2, fp, norm=o.pure_tag)
    assert not errs, errs
    if alt == 2:
        # a tag carries the choice bit exactly when it sits in its alternate
        # bucket: (primary bucket, tag without the bit) of the table entries
        # equals (i1, fp) of the stored keys, as multisets
        b, s = np.nonzero(slots)
        b = b.astype(np.uint64)
        t = slots[b.astype(np.int64), s].astype(np.uint64)
        prim = np.where(t & np.uint64(0x8000), o.alt_map()(b, t), b)
        got = np.stack([prim, t & np.uint64(0x7FFF)], 1)
        want = np.stack([i1.astype(np.uint64), fp.astype(np.uint64)], 1)
        assert np.array_equal(got[np.lexsort(got.T[::-1])], want[np.lexsort(want.T[::-1])])
    half = len(stored) // 2
    out = torch.empty(half, dtype=torch.bool, device="cuda")
    occ1 = f.deleteMany(dev(stored[:half]), out)
    assert host_u8(out).all() and occ1 == occ - half
    assert host_u8(f.containsMany(dev(stored[half:]))).all()
    f.close()


def make_set(cfb, orc, alt, caps):
    cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=16, bucketSize=16, AltBucketPolicy=NAMES[alt])
    s = cfb.CuckooFilterSet(cfg, caps)
    oracles = [orc.OracleFilter(key_bytes=8, bits=16, bucket_size=16, policy=1, max_evictions=500, capacity=int(c),
                                mode=orc.MODE_CONSERVING, alt_policy=alt) for c in caps]
    for i, o in enumerate(oracles):
        assert s.num_buckets[i] == o.nb == cfb.CuckooFilter.calculateNumBuckets(int(caps[i]), 16, NAMES[alt])
    return s, oracles


def set_work(batches):
    keys = np.concatenate([k for _, k in batches])
    offs = np.zeros(len(batches) + 1, np.int64)
    offs[1:] = np.cumsum([len(k) for _, k in batches])
    filt = np.array([f for f, _ in batches], np.int32)
    return dev(keys), torch.from_numpy(offs).cuda(), torch.from_numpy(filt).cuda(), keys


def set_caps(alt):
    # bucket counts that are not powers of two (AddSub: even; Offset: any)
    rng = np.random.default_rng(70 + alt)
    return (16 * rng.integers(300, 5000, 12) + 16 * 3).astype(np.uint64)


@pytest.mark.parametrize("alt", [1, 2])
def test_set_lookups_and_deletes_on_identical_images(cfb, orc, alt):
    """Filter sets with the policy: lookups on images the oracle built equal the
    oracle's, for every probe width; batched deletes remove one copy per key."""
    s, oracles = make_set(cfb, orc, alt, set_caps(alt))
    batches, stored = [], []
    for i, o in enumerate(oracles):
        keys = orc.splitmix64(600 + 10 * alt + i, int(0.9 * o.nb * 16))
        o.insert(keys)
        s.load_table(i, torch.from_numpy(o.table))
        stored.append(keys)
        q = np.concatenate([keys[:700], orc.splitmix64(7000 + i, 500)])
        batches += [(i, q[:300]), (i, q[300:])]
    d_keys, d_offs, d_filt, h_keys = set_work(batches)
    want = np.concatenate([oracles[i].contains(q) for i, q in batches])
    for kpt in (1, 4):
        for w in (1, 4, 8):
            s.set_launch(cfb.SET_CONTAINS, 256, kpt, w)
            out = torch.full((len(h_keys),), 7, dtype=torch.uint8, device="cuda")
            s.contains_async(d_keys, d_offs, d_filt, out)
            s.sync()
            assert np.array_equal(host_u8(out), want), (kpt, w)
    s.clear()
    for i, o in enumerate(oracles):
        s.load_table(i, torch.from_numpy(o.table))
    dels = [(i, k[: len(k) // 2]) for i, k in enumerate(stored)]
    dk, do, df, dh = set_work(dels)
    out = torch.zeros(len(dh), dtype=torch.uint8, device="cuda")
    s.delete_async(dk, do, df, out)
    s.sync()
    assert host_u8(out).all(), "a stored key was not deleted"
    for i, o in enumerate(oracles):
        o.delete(dels[i][1])
        slots = s.table_image(i).numpy().view(np.uint16).reshape(o.nb, 16)
        assert int((slots != 0).sum()) == o.occupied()
        rest = stored[i][len(stored[i]) // 2:]
        i1, i2, fp = o.candidates(rest)
        assert not orc.check_invariants(slots, o.alt_map(), i1, i2, fp, norm=o.pure_tag), i


@pytest.mark.parametrize("alt", [1, 2])
def test_set_inserts_keep_every_filter_invariant(cfb, orc, alt):
    s, oracles = make_set(cfb, orc, alt, set_caps(alt))
    batches, per_filter = [], []
    for i, o in enumerate(oracles):
        keys = orc.splitmix64(650 + 10 * alt + i, int(0.9 * o.nb * 16))
        per_filter.append(keys)
        half = len(keys) // 2
        batches += [(i, keys[:half]), (i, keys[half:])]
    np.random.default_rng(alt).shuffle(batches)
    d_keys, d_offs, d_filt, h_keys = set_work(batches)
    ok = torch.zeros(len(h_keys), dtype=torch.uint8, device="cuda")
    s.insert_async(d_keys, d_offs, d_filt, ok)
    s.sync()
    assert host_u8(ok).all()
    occ = s.occupied()
    for i, o in enumerate(oracles):
        st = s.stats(i)
        slots = s.table_image(i).numpy().view(np.uint16).reshape(o.nb, 16)
        assert st["lost"] == 0 and st["failed"] == 0, (i, st)
        assert int(occ[i]) == int((slots != 0).sum()) == len(per_filter[i]), i
        i1, i2, fp = o.candidates(per_filter[i])
        assert not orc.check_invariants(slots, o.alt_map(), i1, i2, fp, norm=o.pure_tag), i
    out = torch.zeros(len(h_keys), dtype=torch.uint8, device="cuda")
    s.contains_async(d_keys, d_offs, d_filt, out)
    s.sync()
    assert host_u8(out).all(), "false negative"


@pytest.mark.parametrize("alt,policy,max_ev,fill", [(1, 1, 500, 0.97), (2, 0, 500, 0.97), (2, 1, 16, 1.0)])
def test_sorted_insert_one_key_per_call_bit_exact(cfb, orc, alt, policy, max_ev, fill):
    """insertManySorted (segment-staged: one partial segment, 253 buckets) one
    key per call gives the oracle's image."""
    f, o = make(cfb, orc, alt, policy=policy, max_ev=max_ev, cap=4048)
    keys = orc.splitmix64(900 + alt * 10 + policy, int(fill * f.capacity()))
    d = dev(keys)
    out = torch.empty(1, dtype=torch.bool, device="cuda")
    got = np.empty(len(keys), np.uint8)
    for i in range(len(keys)):
        f.insertManySorted(d[i:i + 1], d_output=out)
        got[i] = int(out.item())
    n_ok, want = o.insert(keys, out=True)
    assert np.array_equal(got, want), f"first differing key {int(np.argmax(got != want))}"
    assert np.array_equal(image(f), o.table)


@pytest.mark.parametrize("staging", [2, 3])
@pytest.mark.parametrize("alt", [1, 2])
def test_segment_path_with_partial_last_segment(cfb, orc, alt, staging):
    """~62 500 buckets: 31 segments of 2048 buckets (segment-staged), or 31
    regions of 2048 buckets (region-staged, 64 KiB regions), the last one
    partial.  Staged inserts, lookups and deletes keep every invariant and
    agree with the random path on the same image."""
    f, o = make(cfb, orc, alt, policy=0, cap=1_000_003)
    assert o.nb % 2048 != 0
    f.setOption(cfb.OPT_STAGING, staging)
    if staging == 3:
        f.setOption(cfb.OPT_REGION_BYTES, 1 << 16)
        assert f.getOption(cfb.OPT_REGION_COUNT) == (o.nb - 1) // 2048 + 1
    keys = orc.splitmix64(31 + alt, int(0.95 * f.capacity()))
    d = dev(keys)
    ok_t = torch.empty(len(keys), dtype=torch.bool, device="cuda")
    occ = f.insertMany(d, d_output=ok_t)
    ok = host_u8(ok_t).astype(bool)
    assert occ == ok.sum() == f.countOccupiedSlots() and f.stats()["lost"] == 0
    slots = image(f).view(np.uint16).reshape(o.nb, 16)
    stored = keys[ok]
    i1, i2, fp = o.candidates(stored)
    assert not orc.check_invariants(slots, o.alt_map(), i1, i2, fp, norm=o.pure_tag)
    q = np.concatenate([stored, orc.splitmix64(77, 200_000)])
    seg = host_u8(f.containsMany(dev(q)))
    o.table[:] = image(f)
    assert np.array_equal(seg, o.contains(q))
    assert seg[: len(stored)].all()
    half = len(stored) // 2
    out = torch.empty(half, dtype=torch.bool, device="cuda")
    occ1 = f.deleteMany(dev(stored[:half]), out)
    assert host_u8(out).all() and occ1 == occ - half == f.countOccupiedSlots()
    f.close()
