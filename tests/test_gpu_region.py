"""The region-staged path (cf_region.cuh) against the oracle.

Batches are partitioned by ~16 MiB table region in one pass and applied
region by region so that probes hit L2.  Forced on (CF_OPT_STAGING = region)
for every bucket geometry:

* lookups on an identical table image equal the oracle byte for byte, for
  tables of one region and of many, and with the batch split into many
  workspace chunks at unaligned addresses;
* deletes remove exactly one copy per key; deletes of never-stored keys agree
  with the oracle;
* bulk inserts keep every invariant (no false negatives, (bucket pair, tag)
  multiset conserved, counters equal to the image) with failure counts within
  3 sigma of the oracle's sequential fill;
* the random, segment-staged and region-staged paths return identical lookups.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from test_gpu_parity import _stored_invariants, dev, host_u8, make  # noqa: E402

LOOKUP = [(8, 16, 16), (8, 8, 16), (8, 32, 8), (4, 16, 16), (8, 16, 4), (8, 8, 64), (8, 16, 32), (8, 32, 2),
          (8, 8, 8), (4, 32, 16)]


def small_regions(cfb, f, nbytes=1 << 14):
    """Cut a small table into many regions (at most 256)."""
    f.setOption(cfb.OPT_REGION_BYTES, nbytes)
    return f.getOption(cfb.OPT_REGION_COUNT)


@pytest.mark.parametrize("kb,bits,bs", LOOKUP)
@pytest.mark.parametrize("cap,region_bytes", [(1 << 10, 0), (1 << 18, 0), (1 << 18, 1 << 12), (1 << 22, 1 << 14)])
def test_region_contains_matches_oracle(cfb, orc, kb, bits, bs, cap, region_bytes):
    f, o = make(cfb, orc, kb, bits, bs, 0, 500, cap, "region")
    if region_bytes:
        assert small_regions(cfb, f, region_bytes) > 1
    pos = orc.splitmix64(1, int(0.93 * f.capacity()))
    n_pos = min(len(pos), 1 << 20)
    neg = orc.splitmix64(2, max(4000, n_pos))
    if kb == 4:
        pos, neg = np.unique(pos.astype(np.uint32)), neg.astype(np.uint32)
    o.insert(pos)
    f.load_table(torch.from_numpy(o.table).cuda())
    q = np.concatenate([pos[:n_pos], neg])
    q = q[np.random.default_rng(3).permutation(len(q))]
    got = host_u8(f.containsMany(dev(q)))
    assert np.array_equal(got, o.contains(q, threads=4))


def test_region_contains_chunked_and_unaligned(cfb, orc):
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 22, "region")
    assert small_regions(cfb, f) == 256
    pos = orc.splitmix64(1, int(0.95 * f.capacity()))
    o.insert(pos)
    f.load_table(torch.from_numpy(o.table).cuda())
    f.setOption(cfb.OPT_WORKSPACE_LIMIT, 4 << 20)  # ~160K keys per chunk
    q = np.concatenate([pos[:1_000_000], orc.splitmix64(2, 700_001)])
    buf = dev(np.concatenate([np.zeros(3, np.uint64), q]))
    outbuf = torch.zeros(len(q) + 5, dtype=torch.bool, device="cuda")
    f.containsMany(buf[3:], outbuf[5:])
    assert host_u8(outbuf[:5]).sum() == 0
    assert np.array_equal(host_u8(outbuf[5:]), o.contains(q, threads=4))


@pytest.mark.parametrize("kb,bits,bs", [(8, 16, 16), (8, 32, 8), (8, 8, 16), (4, 16, 16), (8, 16, 4)])
@pytest.mark.parametrize("with_out", [True, False])
def test_region_delete(cfb, orc, kb, bits, bs, with_out):
    f, o = make(cfb, orc, kb, bits, bs, 0, 500, 1 << 20, "region")
    assert small_regions(cfb, f) > 8
    keys = orc.splitmix64(5, int(0.95 * f.capacity()))
    if kb == 4:
        keys = np.unique(keys.astype(np.uint32))
    o.insert(keys)
    f.load_table(torch.from_numpy(o.table).cuda())
    half = keys[: len(keys) // 2]
    out = torch.zeros(len(half), dtype=torch.bool, device="cuda") if with_out else None
    occ = f.deleteMany(dev(half), out)
    if with_out:
        assert host_u8(out).all(), "a stored key was not deleted"
    o.delete(half)
    assert occ == o.occupied() == f.countOccupiedSlots()
    assert f.stats()["removed"] == len(half)
    assert host_u8(f.containsMany(dev(keys[len(keys) // 2:]))).all(), "false negative after delete"
    neg = orc.splitmix64(6, 200_000).astype(keys.dtype)
    out = torch.zeros(len(neg), dtype=torch.bool, device="cuda")
    occ = f.deleteMany(dev(neg), out)
    n_seq, want = o.delete(neg)
    got = host_u8(out)
    assert occ == f.countOccupiedSlots()
    if bits >= 16:
        assert np.array_equal(got, want) and occ == o.occupied()
    else:  # two never-stored keys may compete for one matching copy
        assert abs(int(got.sum()) - n_seq) <= 0.01 * n_seq + 10, (int(got.sum()), n_seq)


def test_region_delete_duplicates_one_copy_each(cfb, orc):
    """k copies of a key need k deletes; the (k+1)-th fails."""
    f, o = make(cfb, orc, 8, 16, 16, 1, 500, 1 << 16, "region")
    base = orc.splitmix64(8, 5000)
    keys = np.concatenate([base, base[:1000], base[:300]])
    assert f.insertMany(dev(keys)) == len(keys)
    out = torch.zeros(len(keys), dtype=torch.bool, device="cuda")
    occ = f.deleteMany(dev(keys), out)
    assert host_u8(out).all() and occ == 0
    out = torch.zeros(300, dtype=torch.bool, device="cuda")
    f.deleteMany(dev(base[:300]), out)
    assert host_u8(out).sum() == 0


BULK = [(8, 16, 16, 0, 1 << 20), (8, 16, 16, 1, 1 << 20), (8, 8, 16, 0, 1 << 20), (8, 32, 8, 1, 1 << 20),
        (4, 16, 16, 1, 1 << 20), (8, 16, 16, 0, 1 << 24), (8, 16, 4, 1, 1 << 16)]


@pytest.mark.parametrize("kb,bits,bs,policy,cap", BULK)
@pytest.mark.parametrize("sorted_", [True, False])
def test_region_bulk_insert_invariants(cfb, orc, kb, bits, bs, policy, cap, sorted_):
    f, o = make(cfb, orc, kb, bits, bs, policy, 500, cap, "region")
    assert small_regions(cfb, f, 1 << 15) > 1
    keys = orc.splitmix64(1, int(0.95 * f.capacity()))
    if kb == 4:
        keys = np.unique(keys.astype(np.uint32))
    d = dev(keys)
    ok_t = torch.zeros(len(keys), dtype=torch.bool, device="cuda")
    occ = (f.insertManySorted if sorted_ else f.insertMany)(d, d_output=ok_t)
    st = f.stats()
    ok = host_u8(ok_t).astype(bool)
    assert occ == ok.sum() == st["occupied"] == f.countOccupiedSlots(), st
    assert st["lost"] == 0
    assert st["primary"] + st["secondary"] + st["evicted_inserts"] == len(keys)
    assert st["failed"] == len(keys) - occ
    assert host_u8(f.containsMany(d[ok_t])).all(), "false negative"
    if cap <= (1 << 20):
        errs = _stored_invariants(f, o, orc, keys[ok])
        assert not errs, errs
        n_seq = o.insert(keys)
        fail_gpu, fail_seq = len(keys) - occ, len(keys) - n_seq
        assert abs(fail_gpu - fail_seq) <= 3 * math.sqrt(max(fail_seq, 1)) + 3, (fail_gpu, fail_seq)


def test_region_insert_chunked(cfb, orc):
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 20, "region")
    small_regions(cfb, f)
    f.setOption(cfb.OPT_WORKSPACE_LIMIT, 1 << 20)
    keys = orc.splitmix64(1, int(0.95 * f.capacity()))
    ok_t = torch.zeros(len(keys), dtype=torch.bool, device="cuda")
    occ = f.insertMany(dev(keys), d_output=ok_t)
    ok = host_u8(ok_t).astype(bool)
    assert occ == ok.sum() == f.countOccupiedSlots() == len(keys)
    errs = _stored_invariants(f, o, orc, keys[ok])
    assert not errs, errs


def test_all_paths_agree(cfb, orc):
    """One table, one query batch, three execution paths: identical bytes."""
    f, o = make(cfb, orc, 8, 16, 16, 0, 500, 1 << 22)
    keys = orc.splitmix64(1, int(0.95 * f.capacity()))
    f.insertMany(dev(keys))
    q = dev(np.concatenate([keys[::3], orc.splitmix64(2, 1_500_000)]))
    outs = []
    for mode in (cfb.STAGING_RANDOM, cfb.STAGING_SEGMENT, cfb.STAGING_REGION):
        f.setOption(cfb.OPT_STAGING, mode)
        outs.append(f.containsMany(q).clone())
    small_regions(cfb, f)
    outs.append(f.containsMany(q).clone())
    assert all(torch.equal(outs[0], x) for x in outs[1:])
