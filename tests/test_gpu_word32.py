"""WordType uint32_t (the reference's word-width comparison geometry,
benchmark/cuckoo_atomics_comparison.cu:13-15).

With 32-bit words the reference scans a bucket from word
(tag & (bs-1)) / tagsPerWord with half as many tags per word, so the slot a
tag lands in differs from the 64-bit-word filter.  The CUDA library keeps its
atomics on 64-bit chunks and only moves the scan start; these tests hold it to
the oracle bit for bit (one key per call, inserts and deletes), pin the
oracle's 32-bit-word mode to the reference's own kernels, and check the bulk
invariants.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from test_gpu_parity import _stored_invariants, dev, host_u8, image  # noqa: E402


def make(cfb, orc, kb, bits, bs, policy, max_ev, cap, staging="auto"):
    cfg = cfb.CuckooConfig(T="uint64" if kb == 8 else "uint32", bitsPerTag=bits, bucketSize=bs,
                           maxEvictions=max_ev, evictionPolicy=cfb.EvictionPolicy(policy), WordType="uint32_t")
    f = cfb.CuckooFilter(cfg, cap)
    if staging != "auto":
        f.setOption(cfb.OPT_STAGING, {"random": 1, "segment": 2, "region": 3}[staging])
    o = orc.OracleFilter(key_bytes=kb, bits=bits, bucket_size=bs, word_bytes=4, policy=policy,
                         max_evictions=max_ev, capacity=cap, mode=orc.MODE_CONSERVING)
    assert f.getNumBuckets() == o.nb
    return f, o


SEQ = [
    # key_bytes, bits, bs, policy, max_ev, capacity, fill
    (8, 8, 16, 1, 500, 1 << 12, 0.97),
    (8, 8, 16, 0, 500, 1 << 12, 0.97),
    (8, 16, 16, 0, 500, 1 << 12, 0.97),
    (8, 16, 16, 1, 16, 1 << 12, 1.00),
    (4, 16, 16, 1, 500, 1 << 12, 0.97),
    (8, 32, 8, 0, 16, 1 << 11, 1.00),
]


@pytest.mark.parametrize("kb,bits,bs,policy,max_ev,cap,fill", SEQ)
def test_sequential_image_bit_exact(cfb, orc, kb, bits, bs, policy, max_ev, cap, fill):
    f, o = make(cfb, orc, kb, bits, bs, policy, max_ev, cap)
    keys = orc.splitmix64(700 + bits + bs + policy, int(fill * f.capacity()))
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
    assert f.stats()["occupied"] == n_ok == f.countOccupiedSlots()


def test_word_width_moves_slots(cfb, orc):
    """Same keys, 32- against 64-bit words: same occupancy, different images."""
    o4 = orc.OracleFilter(key_bytes=8, bits=8, bucket_size=16, word_bytes=4, capacity=1 << 12)
    o8 = orc.OracleFilter(key_bytes=8, bits=8, bucket_size=16, word_bytes=8, capacity=1 << 12)
    keys = orc.splitmix64(9, 3000)
    o4.insert(keys)
    o8.insert(keys)
    assert o4.occupied() == o8.occupied() and not np.array_equal(o4.table, o8.table)


@pytest.mark.parametrize("cfg_key,cap", [((8, 8, 16, 1, 500), 1 << 12), ((8, 8, 16, 0, 500), 1 << 12),
                                         ((8, 16, 16, 1, 500), 1 << 12), ((8, 16, 16, 0, 16), 1 << 12)])
def test_reference_kernels_with_32bit_words_match_oracle(cfb, orc, cfg_key, cap):
    """The reference's own kernels with WordType uint32_t, one key per launch,
    against the oracle's 32-bit-word reference mode up to the first failed chain."""
    if orc.ref_gpu() is None:
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    from test_gpu_parity import _ref_image

    kb, bits, bs, policy, max_ev = cfg_key
    ref = orc.RefGpuFilter(kb, bits, bs, policy, max_ev, cap, word_bytes=4)
    try:
        o = orc.OracleFilter(key_bytes=kb, bits=bits, bucket_size=bs, word_bytes=4, policy=policy,
                             max_evictions=max_ev, capacity=cap, mode=orc.MODE_REFERENCE)
        assert ref.num_buckets() == o.nb
        keys = orc.splitmix64(900 + bits + policy, int(0.97 * cap))
        d = dev(keys)
        prev = 0
        for i in range(len(keys)):
            occ = ref.insert(d[i:i + 1].data_ptr(), 1)
            ok = occ - prev
            prev = occ
            want = o.insert(keys[i:i + 1])
            assert ok == want, i
            if want == 0 or i == len(keys) - 1 or i % 512 == 0:
                assert np.array_equal(_ref_image(cfb, ref, kb, bits, bs), o.table), f"image differs after key {i}"
            if want == 0:
                break
    finally:
        ref.close()


@pytest.mark.parametrize("kb,bits,bs", [(8, 8, 16), (8, 16, 16), (8, 32, 8)])
def test_sequential_delete_bit_exact(cfb, orc, kb, bits, bs):
    f, o = make(cfb, orc, kb, bits, bs, 0, 500, 1 << 12)
    keys = orc.splitmix64(57, int(0.9 * f.capacity()))
    o.insert(keys)
    f.load_table(torch.from_numpy(o.table).cuda())
    dels = np.concatenate([keys[::3], orc.splitmix64(58, 200), keys[:50]])
    d = dev(dels)
    out = torch.empty(1, dtype=torch.bool, device="cuda")
    got = np.empty(len(dels), np.uint8)
    for i in range(len(dels)):
        f.deleteMany(d[i:i + 1], out)
        got[i] = int(out.item())
    _, want = o.delete(dels)
    assert np.array_equal(got, want)
    assert np.array_equal(image(f), o.table)


@pytest.mark.parametrize("staging", ["random", "segment", "region"])
@pytest.mark.parametrize("kb,bits,bs,policy", [(8, 8, 16, 1), (8, 16, 16, 0)])
def test_bulk_insert_and_delete_invariants(cfb, orc, kb, bits, bs, policy, staging):
    f, o = make(cfb, orc, kb, bits, bs, policy, 500, 1 << 20, staging)
    keys = orc.splitmix64(1, int(0.95 * f.capacity()))
    d = dev(keys)
    ok_t = torch.empty(len(keys), dtype=torch.bool, device="cuda")
    occ = f.insertManySorted(d, d_output=ok_t) if staging == "segment" else f.insertMany(d, d_output=ok_t)
    ok = host_u8(ok_t).astype(bool)
    st = f.stats()
    assert occ == ok.sum() == st["occupied"] == f.countOccupiedSlots()
    assert st["lost"] == 0 and st["failed"] == len(keys) - ok.sum()
    assert host_u8(f.containsMany(d[torch.from_numpy(ok).cuda()])).all(), "false negative"
    errs = _stored_invariants(f, o, orc, keys[ok])
    assert not errs, errs
    stored = keys[ok]
    half = len(stored) // 2
    out = torch.empty(half, dtype=torch.bool, device="cuda")
    occ1 = f.deleteMany(dev(stored[:half]), out)
    assert host_u8(out).all() and occ1 == occ - half
    assert host_u8(f.containsMany(dev(stored[half:]))).all()
