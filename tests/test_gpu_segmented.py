"""The segment-staged path (insertManySorted; containsMany/deleteMany on large
batches) against the oracle.

* one key per call: insertManySorted produces the oracle's table image bit for
  bit (the same per-key steps as the plain path, evictions and failed chains
  included);
* bulk inserts: the structural invariants and failure counts within 3 sigma of
  the oracle's sequential fill;
* lookups forced through the segment path equal the oracle on an identical
  image, for every bucket geometry, with and without the segmented second round,
  and with the batch split into many workspace chunks;
* deletes forced through the segment path: exactly one copy per key.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from test_gpu_parity import _stored_invariants, dev, host_u8, image, make  # noqa: E402


def force_segmented(cfb, f, round2_segmented=True):
    """Always take the segment path; second round segment-staged or random."""
    f.setOption(cfb.OPT_SEGMENTED_MIN_KEYS, 1)
    f.setOption(cfb.OPT_ROUND2_SEGMENTED_MIN_KEYS, 1 if round2_segmented else cfb.NEVER)


SEQ = [
    (8, 16, 16, 0, 500, 1 << 12, 0.97),
    (8, 16, 16, 1, 16, 1 << 12, 1.00),
    (8, 32, 8, 1, 16, 1 << 11, 1.00),
    (8, 8, 16, 0, 500, 1 << 12, 0.97),
    (4, 16, 16, 1, 500, 1 << 12, 0.97),
    (8, 16, 64, 1, 500, 1 << 12, 0.97),
    (8, 16, 128, 0, 500, 1 << 12, 0.97),
]


@pytest.mark.parametrize("kb,bits,bs,policy,max_ev,cap,fill", SEQ)
def test_sorted_insert_one_key_per_call_bit_exact(cfb, orc, kb, bits, bs, policy, max_ev, cap, fill):
    f, o = make(cfb, orc, kb, bits, bs, policy, max_ev, cap)
    keys = orc.splitmix64(200 + bits + bs + policy, int(fill * f.capacity()))
    if kb == 4:
        keys = keys.astype(np.uint32)
    d = dev(keys)
    out = torch.empty(1, dtype=torch.bool, device="cuda")
    got = np.empty(len(keys), np.uint8)
    for i in range(len(keys)):
        f.insertManySorted(d[i:i + 1], d_output=out)
        got[i] = int(out.item())
    n_ok, want = o.insert(keys, out=True)
    assert np.array_equal(got, want), f"first differing key {int(np.argmax(got != want))}"
    assert np.array_equal(image(f), o.table)
    assert f.stats()["lost"] == 0


BULK = [(8, 16, 16, 0, 1 << 20, 0.95), (8, 16, 16, 1, 1 << 20, 0.95), (8, 8, 16, 0, 1 << 20, 0.95),
        (8, 32, 8, 1, 1 << 20, 0.95), (8, 32, 8, 0, 1 << 20, 0.95), (4, 16, 16, 1, 1 << 20, 0.95),
        (8, 16, 16, 0, 1 << 24, 0.95), (8, 8, 64, 0, 1 << 20, 0.95), (8, 32, 2, 0, 1 << 18, 0.80),
        (8, 16, 4, 1, 1 << 16, 0.90), (8, 16, 64, 1, 1 << 20, 0.95), (8, 16, 128, 0, 1 << 20, 0.95)]


@pytest.mark.parametrize("kb,bits,bs,policy,cap,fill", BULK)
@pytest.mark.parametrize("with_out", [True, False])
def test_sorted_bulk_insert_invariants(cfb, orc, kb, bits, bs, policy, cap, fill, with_out):
    f, o = make(cfb, orc, kb, bits, bs, policy, 500, cap)
    keys = orc.splitmix64(1, int(fill * f.capacity()))
    if kb == 4:
        keys = np.unique(keys.astype(np.uint32))
    d = dev(keys)
    ok_t = torch.zeros(len(keys), dtype=torch.bool, device="cuda") if with_out else None
    occ = f.insertManySorted(d, d_output=ok_t)
    st = f.stats()
    assert occ == st["occupied"] == f.countOccupiedSlots()
    assert st["lost"] == 0
    assert st["primary"] + st["secondary"] + st["evicted_inserts"] == len(keys)
    assert st["failed"] == len(keys) - occ
    if with_out:
        ok = host_u8(ok_t).astype(bool)
        assert ok.sum() == occ
        stored = keys[ok]
        assert host_u8(f.containsMany(d[ok_t])).all(), "false negative"
        if cap <= (1 << 20):
            errs = _stored_invariants(f, o, orc, stored)
            assert not errs, errs
    else:
        assert occ == len(keys) or st["failed"] > 0
        if st["failed"] == 0:
            assert host_u8(f.containsMany(d)).all()
    if cap <= (1 << 20):
        n_seq = o.insert(keys)
        fail_gpu, fail_seq = len(keys) - occ, len(keys) - n_seq
        sigma = math.sqrt(max(fail_seq, 1))
        assert abs(fail_gpu - fail_seq) <= 3 * sigma + 3, (fail_gpu, fail_seq)
        if policy == orc.POLICY_BFS:
            # BFS resolves most keys with one eviction; a search that skips
            # candidates falls back to DFS walks and inflates the ratio
            seq = dict(zip(orc.STAT_NAMES, o.stats.tolist()))
            r_seq = seq["evictions"] / max(seq["evicted_inserts"], 1)
            r_gpu = st["evictions"] / max(st["evicted_inserts"], 1)
            assert r_gpu <= 1.5 * r_seq + 0.25, (r_gpu, r_seq, st, seq)


@pytest.mark.parametrize("sorted_", [True, False])
def test_over_capacity_counters_stay_exact(cfb, orc, sorted_):
    """2-slot buckets filled past what they can hold: most late inserts fail and
    run full eviction walks that cross.  The occupancy counter must equal the
    table's occupied slots, and tags dropped by crossing walks stay rare."""
    f, o = make(cfb, orc, 8, 32, 2, 1, 500, 1 << 16)
    hk = orc.splitmix64(4, int(0.98 * f.capacity()))
    keys = dev(hk)
    occ = f.insertManySorted(keys) if sorted_ else f.insertMany(keys)
    st = f.stats()
    assert occ == st["occupied"] == f.countOccupiedSlots(), st
    # keys that end up unstored: rejected (failed) or displaced by a crossing walk (lost)
    n_seq = o.insert(hk)
    seq_fail = len(hk) - n_seq
    assert seq_fail > 0
    unstored = st["failed"] + st["lost"]
    assert abs(unstored - seq_fail) <= 0.25 * seq_fail + 3 * math.sqrt(seq_fail), (st, seq_fail)


def test_sorted_insert_chunked_equals_unchunked_counts(cfb, orc):
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 20)
    f.setOption(cfb.OPT_WORKSPACE_LIMIT, 1 << 20)  # 1 MiB workspace: ~40K keys per chunk
    keys = orc.splitmix64(1, int(0.95 * f.capacity()))
    d = dev(keys)
    ok_t = torch.zeros(len(keys), dtype=torch.bool, device="cuda")
    occ = f.insertManySorted(d, d_output=ok_t)
    ok = host_u8(ok_t).astype(bool)
    assert occ == ok.sum() == f.countOccupiedSlots() == len(keys)
    assert f.getOption(cfb.OPT_WORKSPACE_BYTES) <= 2 << 20
    errs = _stored_invariants(f, o, orc, keys[ok])
    assert not errs, errs


def test_workspace_default_is_automatic_and_holds_the_whole_batch(cfb, orc):
    """The default workspace limit is automatic: a batch that fits the free
    device memory runs in one chunk (16 bytes per key without per-key results,
    about 24 with them), and the workspace is kept for later calls."""
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 25)
    try:
        assert f.getOption(cfb.OPT_WORKSPACE_LIMIT) == 0
        n = 1 << 23  # two batches fill the table to half its capacity
        keys = orc.splitmix64(91, n)
        occ = f.insertManySorted(dev(keys))
        ws = f.getOption(cfb.OPT_WORKSPACE_BYTES)
        assert occ == n and ws >= 16 * n
        ok_t = torch.zeros(n, dtype=torch.bool, device="cuda")
        f.insertManySorted(dev(orc.splitmix64(92, n)), d_output=ok_t)
        assert host_u8(ok_t).all() and f.getOption(cfb.OPT_WORKSPACE_BYTES) >= 24 * n
        assert f.countOccupiedSlots() == 2 * n
    finally:
        f.close()


def test_repeated_batch_reuses_the_workspace_in_one_chunk(cfb, orc):
    """A batch that fits the workspace an earlier call left is not split: the
    same fill, repeated on the cleared table, launches exactly the kernels the
    first one did (a split would add a second radix / segment chain)."""
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 22)
    try:
        keys = dev(orc.splitmix64(93, int(0.95 * f.capacity())))
        counts = []
        for _ in range(3):
            f.clear()
            before = cfb.launch_count()
            assert f.insertManySorted(keys) == keys.numel()
            counts.append(cfb.launch_count() - before)
        assert counts[0] == counts[1] == counts[2], counts
    finally:
        f.close()


LOOKUP = [(8, 16, 16), (8, 8, 16), (8, 32, 8), (4, 16, 16), (8, 16, 4), (8, 8, 64), (8, 16, 32), (8, 32, 2),
          (8, 8, 8), (4, 32, 16)]


@pytest.mark.parametrize("kb,bits,bs", LOOKUP)
@pytest.mark.parametrize("round2_segmented", [True, False])
@pytest.mark.parametrize("cap", [1 << 10, 1 << 18])
def test_segmented_contains_matches_oracle(cfb, orc, kb, bits, bs, round2_segmented, cap):
    f, o = make(cfb, orc, kb, bits, bs, 0, 500, cap)
    pos = orc.splitmix64(1, int(0.93 * f.capacity()))
    neg = orc.splitmix64(2, max(4000, len(pos)))
    if kb == 4:
        pos, neg = pos.astype(np.uint32), neg.astype(np.uint32)
    o.insert(pos)
    f.load_table(torch.from_numpy(o.table).cuda())
    force_segmented(cfb, f, round2_segmented)
    q = np.concatenate([pos, neg])
    rng = np.random.default_rng(3)
    q = q[rng.permutation(len(q))]
    got = host_u8(f.containsMany(dev(q)))
    assert np.array_equal(got, o.contains(q, threads=4))


def test_segmented_contains_chunked_and_unaligned(cfb, orc):
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 18)
    pos = orc.splitmix64(1, int(0.95 * f.capacity()))
    o.insert(pos)
    f.load_table(torch.from_numpy(o.table).cuda())
    force_segmented(cfb, f)
    f.setOption(cfb.OPT_WORKSPACE_LIMIT, 1 << 20)
    q = np.concatenate([pos, orc.splitmix64(2, 300_001)])
    buf = dev(np.concatenate([np.zeros(3, np.uint64), q]))
    outbuf = torch.zeros(len(q) + 5, dtype=torch.bool, device="cuda")
    f.containsMany(buf[3:], outbuf[5:])
    got = host_u8(outbuf[5:])
    assert host_u8(outbuf[:5]).sum() == 0
    assert np.array_equal(got, o.contains(q, threads=4))


@pytest.mark.parametrize("kb,bits,bs,round2_segmented", [(8, 16, 16, True), (8, 16, 16, False), (8, 32, 8, True),
                                                         (8, 8, 16, False), (4, 16, 16, True)])
def test_segmented_delete(cfb, orc, kb, bits, bs, round2_segmented):
    f, o = make(cfb, orc, kb, bits, bs, 0, 500, 1 << 18)
    keys = orc.splitmix64(5, int(0.95 * f.capacity()))
    if kb == 4:
        keys = np.unique(keys.astype(np.uint32))
    o.insert(keys)
    f.load_table(torch.from_numpy(o.table).cuda())
    force_segmented(cfb, f, round2_segmented)
    half = keys[: len(keys) // 2]
    out = torch.zeros(len(half), dtype=torch.bool, device="cuda")
    occ = f.deleteMany(dev(half), out)
    assert host_u8(out).all(), "a stored key was not deleted"
    o.delete(half)
    assert occ == o.occupied() == f.countOccupiedSlots()
    assert host_u8(f.containsMany(dev(keys[len(keys) // 2:]))).all(), "false negative after delete"
    # keys never stored: a delete succeeds only on a false-positive tag match, as in the reference
    neg = orc.splitmix64(6, 200_000).astype(keys.dtype)
    out = torch.zeros(len(neg), dtype=torch.bool, device="cuda")
    occ = f.deleteMany(dev(neg), out)
    n_seq, want = o.delete(neg)
    got = host_u8(out)
    assert occ == f.countOccupiedSlots()
    if bits >= 16:
        assert got.sum() == n_seq and occ == o.occupied()
        assert np.array_equal(got, want)
    else:
        # 8-bit tags: ~12% of never-stored keys match a stored tag, and two such
        # deletes may compete for one copy, so which key wins depends on order
        assert abs(int(got.sum()) - n_seq) <= 0.01 * n_seq + 10, (int(got.sum()), n_seq)


def test_segmented_paths_agree_with_plain_paths(cfb, orc):
    """Same batch through the plain and the segment-staged lookup: identical bytes."""
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 20)
    keys = orc.splitmix64(1, int(0.95 * f.capacity()))
    f.insertMany(dev(keys))
    q = dev(np.concatenate([keys[::3], orc.splitmix64(2, 500_000)]))
    f.setOption(cfb.OPT_SEGMENTED_MIN_KEYS, cfb.NEVER)
    plain = f.containsMany(q).clone()
    force_segmented(cfb, f)
    seg = f.containsMany(q)
    assert torch.equal(plain, seg)


def test_insertMany_stages_batches_of_at_least_one_key_per_bucket(cfb, orc):
    """insertMany picks the segment path from one key per bucket on (many
    launches per call) and probes at random below it (one launch); both keep
    the invariants."""
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 18)  # 16384 buckets
    nb = f.getNumBuckets()
    keys = orc.splitmix64(44, int(0.9 * f.capacity()))
    small, big = keys[: nb // 2], keys[nb // 2:]
    c0 = cfb.launch_count()
    f.insertMany(dev(small))
    c1 = cfb.launch_count()
    f.insertMany(dev(big))
    c2 = cfb.launch_count()
    assert c1 - c0 <= 2 and c2 - c1 >= 8, (c1 - c0, c2 - c1)
    st = f.stats()
    assert st["failed"] == 0 and st["lost"] == 0 and st["occupied"] == len(keys) == f.countOccupiedSlots()
    assert not _stored_invariants(f, o, orc, keys)
    assert host_u8(f.containsMany(dev(keys))).all()
    # the option moves the threshold: never stage
    f.clear()
    f.setOption(cfb.OPT_SEGMENTED_MIN_KEYS, cfb.NEVER)
    c3 = cfb.launch_count()
    f.insertMany(dev(big))
    assert cfb.launch_count() - c3 <= 2


def test_round1_cap_option(cfb, orc):
    """CF_OPT_ROUND1_CAP on a 0.95 sorted fill: automatic (13 of 16 slots in
    the first round, a third round at the primary bucket), the reference's
    primary-first order (16) and an explicit 12 all keep every invariant; the
    automatic cap sends more keys to their alternate bucket and leaves fewer
    for eviction than the primary-first order."""
    res = {}
    for capv in (0, 16, 12):
        f, o = make(cfb, orc, 8, 16, 16, 1, 500, 1 << 20)
        f.setOption(cfb.OPT_ROUND1_CAP, capv)
        assert f.getOption(cfb.OPT_ROUND1_CAP) == capv
        keys = orc.splitmix64(77, int(0.95 * f.capacity()))
        d = dev(keys)
        ok_t = torch.empty(len(keys), dtype=torch.bool, device="cuda")
        occ = f.insertManySorted(d, d_output=ok_t)
        st = f.stats()
        ok = host_u8(ok_t).astype(bool)
        assert occ == ok.sum() == f.countOccupiedSlots() and st["lost"] == 0, (capv, st)
        assert st["primary"] + st["secondary"] + st["evicted_inserts"] == len(keys)
        assert host_u8(f.containsMany(d[ok_t])).all(), "false negative"
        errs = _stored_invariants(f, o, orc, keys[ok])
        assert not errs, (capv, errs)
        res[capv] = st
        f.close()
    assert res[0]["secondary"] > res[16]["secondary"]
    assert res[0]["evicted_inserts"] < res[16]["evicted_inserts"], (res[0], res[16])
    f, _ = make(cfb, orc, 8, 16, 16, 1, 500, 1 << 12)
    with pytest.raises(cfb.CuckooError):
        f.setOption(cfb.OPT_ROUND1_CAP, 17)
    f.close()


def test_insert_into_known_empty_table_keeps_every_earlier_write(cfb, orc):
    """The first segment round of an insert into a table the library knows to
    be all zeros (just created or cleared) stages zeroed segments instead of
    loading them.  Every call that may write the table drops that knowledge:
    a second insert, an insert on the random path, a delete, a table load and
    a chunked batch must all keep what is already stored."""
    cap = 1 << 22
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, cap)
    try:
        def present(keys):
            return host_u8(f.containsMany(dev(keys))).all()

        a = orc.splitmix64(301, int(0.4 * cap))
        b = orc.splitmix64(302, int(0.4 * cap))
        # fresh table: sorted insert, then a second sorted insert
        assert f.insertManySorted(dev(a)) == len(a)
        assert f.insertManySorted(dev(b)) == len(a) + len(b)
        assert present(a) and present(b) and f.countOccupiedSlots() == len(a) + len(b)
        # cleared table: only the new keys, counters from zero
        f.clear()
        assert f.countOccupiedSlots() == 0
        assert f.insertManySorted(dev(b)) == len(b) == f.countOccupiedSlots()
        assert present(b)
        # a small random-path insert, then a sorted one
        f.clear()
        small = orc.splitmix64(303, 1000)
        f.setOption(cfb.OPT_STAGING, cfb.STAGING_RANDOM)
        f.insertMany(dev(small))
        f.setOption(cfb.OPT_STAGING, cfb.STAGING_AUTO)
        f.insertManySorted(dev(a))
        assert present(small) and present(a) and f.countOccupiedSlots() == len(small) + len(a)
        # a delete on a cleared table, then a sorted insert
        f.clear()
        f.deleteMany(dev(small))
        assert f.insertManySorted(dev(a)) == len(a) and present(a)
        # a loaded table image, then a sorted insert
        o.insert(b)
        f.load_table(torch.from_numpy(o.table).cuda())
        f.insertManySorted(dev(a))
        assert present(b) and present(a) and f.countOccupiedSlots() == len(a) + len(b)
    finally:
        f.close()
    # a batch in several chunks on a new table: only the first chunk is staged as zeros
    g, _ = make(cfb, orc, 8, 16, 16, 0, 500, cap)
    try:
        g.setOption(cfb.OPT_WORKSPACE_LIMIT, 16 << 20)  # about 1 M keys per chunk
        both = np.concatenate([a, b])
        assert g.insertManySorted(dev(both)) == len(both) == g.countOccupiedSlots()
        assert g.getOption(cfb.OPT_WORKSPACE_BYTES) <= 16 << 20  # the batch ran in chunks
        assert host_u8(g.containsMany(dev(both))).all()
        assert g.stats()["failed"] == 0 and g.stats()["lost"] == 0
    finally:
        g.close()
