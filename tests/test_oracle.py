"""The oracle is pinned before it is trusted (CPU only).

* hashing / bucket derivation against the golden vectors produced by the
  reference's own compiled ``XorAltBucketPolicy`` (tests/golden/make_golden.py);
* the same, live, against ``oracle/_ref/libref_host.so`` when it is present;
* the sequential insert/delete restatement against the reference's documented
  behaviour and the structural invariants.
"""
from __future__ import annotations

import numpy as np
import pytest


def _cases(golden):
    i = 0
    while f"c{i}_meta" in golden:
        kb, bits, bs, cap, nb = (int(x) for x in golden[f"c{i}_meta"])
        yield i, kb, bits, bs, cap, nb
        i += 1


def test_golden_candidates(golden, orc):
    n_cases = 0
    for i, kb, bits, bs, cap, nb in _cases(golden):
        f = orc.OracleFilter(key_bytes=kb, bits=bits, bucket_size=bs, capacity=cap) if nb < (1 << 28) else None
        p = orc.Params(kb, bits, bs, 8, 1, 500, nb)
        keys = golden[f"c{i}_keys"]
        i1 = np.empty(len(keys), np.uint64)
        i2 = np.empty(len(keys), np.uint64)
        fp = np.empty(len(keys), np.uint32)
        import ctypes as C

        orc.lib().cfo_candidates(C.byref(p), keys.ctypes.data, len(keys), i1.ctypes.data, i2.ctypes.data,
                                 fp.ctypes.data)
        assert np.array_equal(i1, golden[f"c{i}_i1"]), f"case {i}: i1"
        assert np.array_equal(i2, golden[f"c{i}_i2"]), f"case {i}: i2"
        assert np.array_equal(fp, golden[f"c{i}_fp"]), f"case {i}: fp"
        hashes = [orc.xxhash64(int(k), kb) for k in keys[:64]]
        assert hashes == [int(h) for h in golden[f"c{i}_hash"][:64]]
        assert orc.num_buckets(cap, bs) == nb
        del f
        n_cases += 1
    assert n_cases >= 10


def test_golden_tag_hashes(golden, orc):
    for bits in (8, 16, 32):
        tags = golden[f"tag{bits}"]
        want = golden[f"taghash{bits}"]
        got = np.array([orc.xxhash64(int(t), bits // 8) for t in tags], dtype=np.uint64)
        assert np.array_equal(got, want), bits


def test_golden_num_buckets(golden, orc):
    for cap, bs, nb in golden["num_buckets"]:
        assert orc.num_buckets(int(cap), int(bs)) == int(nb), (cap, bs)


def test_golden_fp_zero_maps_to_one(golden):
    """Keys whose masked fingerprint is 0 are stored with tag 1 (bucket_policies.cuh:53)."""
    found = 0
    for i, kb, bits, bs, cap, nb in _cases(golden):
        h = golden[f"c{i}_hash"]
        mask = (1 << bits) - 1 if bits < 32 else 0xFFFFFFFF
        zero = ((h >> np.uint64(32)) & np.uint64(mask)) == 0
        if zero.any():
            assert (golden[f"c{i}_fp"][zero] == 1).all()
            found += int(zero.sum())
    assert found > 0


def test_known_answers_for_keys_1_and_42(orc):
    """Known answers computed from the reference headers for key 1 and key 42
    at 16-bit tags, bucket size 16, 2^16 buckets."""
    f = orc.OracleFilter(capacity=1 << 20)
    assert f.nb == 65536
    assert orc.xxhash64(1, 8) == 0x9F29CB17A2A49995
    i1, i2, fp = f.candidates([1, 42])
    assert list(i1) == [39317, 17235] and list(i2) == [24287, 21006] and list(fp) == [51991, 32879]


def test_live_reference_hashing(orc):
    """Against the reference compiled from its sources (skipped where they are absent)."""
    if orc.ref_host() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    keys = orc.splitmix64(77, 200_000)
    for kb in (8, 4):
        for bits, bs in ((8, 16), (16, 16), (32, 8), (16, 4), (8, 64)):
            f = orc.OracleFilter(key_bytes=kb, bits=bits, bucket_size=bs, capacity=1 << 22)
            k = keys if kb == 8 else keys.astype(np.uint32)
            a = f.candidates(k)
            b = orc.ref_candidates(kb, bits, bs, f.nb, k)
            for x, y in zip(a, b):
                assert np.array_equal(x, y), (kb, bits, bs)


# ------------------------------------------------------- sequential semantics


def _slots(f):
    return f.slots()


def test_insert_first_empty_slot_rule(orc):
    """tryInsertAtBucket scans words from (fp & (bs-1)) / tagsPerWord and takes
    the lowest empty lane (CuckooFilter.cuh:859-904)."""
    f = orc.OracleFilter(bits=16, bucket_size=16, capacity=1 << 12, policy=orc.POLICY_DFS)
    keys = orc.splitmix64(3, 1)
    i1, i2, fp = f.candidates(keys)
    f.insert(keys)
    s = _slots(f)
    start = (int(fp[0]) & 15) // 4 * 4
    assert s[int(i1[0]), start] == fp[0]
    assert np.count_nonzero(s) == 1


def test_sequential_fill_invariants(orc):
    for bits, bs in ((16, 16), (8, 16), (32, 8)):
        for pol in (orc.POLICY_BFS, orc.POLICY_DFS):
            f = orc.OracleFilter(bits=bits, bucket_size=bs, capacity=1 << 14, policy=pol)
            keys = orc.splitmix64(11, int(0.95 * (1 << 14)))
            n, ok = f.insert(keys, out=True)
            assert n == ok.sum()
            assert f.occupied() == n
            stored = keys[ok.astype(bool)]
            assert f.contains(stored).all(), "false negative after insert"
            i1, i2, fp = f.candidates(stored)
            alt = orc.alt_vectorized(bits, f.nb) if bits <= 16 else (lambda b, t: np.array(
                [f.alt_bucket(int(x), int(y)) for x, y in zip(b, t)], dtype=np.uint64))
            errs = orc.check_invariants(f.slots(), alt, i1, i2, fp)
            assert not errs, errs


def test_reference_and_conserving_modes_agree_until_first_failure(orc):
    """The two failure modes make identical choices until a DFS chain fails."""
    for bits, bs in ((16, 16), (32, 8)):
        keys = orc.splitmix64(5, 1 << 12)
        ref = orc.OracleFilter(bits=bits, bucket_size=bs, capacity=1 << 12, policy=orc.POLICY_DFS,
                               max_evictions=16, mode=orc.MODE_REFERENCE)
        con = orc.OracleFilter(bits=bits, bucket_size=bs, capacity=1 << 12, policy=orc.POLICY_DFS,
                               max_evictions=16, mode=orc.MODE_CONSERVING)
        first_fail = None
        for i, k in enumerate(keys):
            r1 = ref.insert([k])
            r2 = con.insert([k])
            assert r1 == r2
            if r1 == 0:
                first_fail = i
                break
            assert np.array_equal(ref.table, con.table), i
        assert first_fail is not None, "filter never overflowed"
        # after the failure, the conserving table equals the pre-insert table
        snap = con.table.copy()
        con.insert([keys[first_fail]])
        assert np.array_equal(con.table, snap)


def test_conserving_failure_restores_table(orc):
    f = orc.OracleFilter(bits=32, bucket_size=8, capacity=1 << 10, policy=orc.POLICY_DFS, max_evictions=8)
    keys = orc.splitmix64(21, 1 << 11)
    failures = 0
    for k in keys:
        snap = f.table.copy()
        if f.insert([k]) == 0:
            failures += 1
            assert np.array_equal(f.table, snap)
    assert failures > 0


def test_delete_one_copy_per_key(orc):
    f = orc.OracleFilter(bits=16, bucket_size=16, capacity=10000)
    keys = np.array([1, 1, 1, 2, 2, 3], dtype=np.uint64)
    assert f.insert(keys) == 6
    n, out = f.delete(np.array([1, 1, 1, 1], dtype=np.uint64))
    assert n == 3 and list(out) == [1, 1, 1, 0]
    assert f.occupied() == 3
    assert list(f.contains(np.array([1, 2, 3], dtype=np.uint64))) == [0, 1, 1]


def test_multithreaded_port_matches_sequential_lookups(orc):
    f = orc.OracleFilter(bits=16, bucket_size=16, capacity=1 << 16, policy=orc.POLICY_BFS)
    keys = orc.splitmix64(1, int(0.9 * (1 << 16)))
    f.insert(keys)
    q = np.concatenate([keys[:5000], orc.splitmix64(2, 5000)])
    assert np.array_equal(f.contains(q, threads=1), f.contains(q, threads=4))


def test_multithreaded_insert_has_no_false_negatives(orc):
    import ctypes as C

    f = orc.OracleFilter(bits=16, bucket_size=16, capacity=1 << 16, policy=orc.POLICY_BFS)
    keys = orc.splitmix64(9, int(0.95 * (1 << 16)))
    out = np.empty(len(keys), np.uint8)
    n = orc.lib().cfo_insert_mt(C.byref(f.p), f.table.ctypes.data, keys.ctypes.data, len(keys), out.ctypes.data, 4)
    assert n == out.sum() == f.occupied()
    assert f.contains(keys[out.astype(bool)]).all()
