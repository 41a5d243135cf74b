"""The AddSub and Offset alternate-bucket policies (reference
include/bucket_policies.cuh:95-350) in the oracle, pinned to the reference's
own policy code compiled from its headers (oracle/_ref/libref_host.so).

CPU only: candidates, alternate buckets (with the Offset policy's choice-bit
flip), bucket counts, the involution property, and the sequential filter's
behaviour (every stored key found, deletes remove one copy, the bucket-pair /
tag multiset invariant)."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def ref(orc):
    if orc.ref_host() is None:
        pytest.skip("oracle/_ref/libref_host.so not built")
    return orc


POLICIES = [1, 2]  # ALT_ADDSUB, ALT_OFFSET


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("kb,bits", [(8, 16), (8, 8), (8, 32), (4, 16)])
@pytest.mark.parametrize("nb", [1 << 12, 6_000_002, 999_999 * 2, 65_536 + 2])
def test_candidates_match_reference(ref, policy, kb, bits, nb):
    if policy == 1 and nb % 2:
        pytest.skip("AddSub needs an even bucket count")
    o = ref.OracleFilter(key_bytes=kb, bits=bits, bucket_size=16, alt_policy=policy, capacity=16)
    o.nb = nb
    o.p.num_buckets = nb
    keys = ref.splitmix64(40 + bits + policy, 20_000)
    keys = np.concatenate([keys, np.array([0, 1, 2**32 - 1, 2**64 - 1], np.uint64)])
    if kb == 4:
        keys = keys.astype(np.uint32)
    got = o.candidates(keys)
    want = ref.ref_candidates_policy(policy, kb, bits, nb, keys)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    i1, i2, fp = got
    assert (i1 < nb).all() and (i2 < nb).all() and (fp != 0).all()
    if policy == 1:
        assert (i1 < nb // 2).all() and (i2 >= nb // 2).all()
    else:
        assert (fp < (1 << (bits - 1))).all()  # choice bit 0 in the primary bucket


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("bits", [8, 16, 32])
def test_alternate_bucket_and_tag_match_reference(ref, policy, bits):
    nb = 1_000_006
    o = ref.OracleFilter(bits=bits, bucket_size=16, alt_policy=policy, capacity=16)
    o.nb = nb
    o.p.num_buckets = nb
    rng = np.random.default_rng(bits)
    b = rng.integers(0, nb, 5000).astype(np.uint64)
    t = rng.integers(1, 1 << bits, 5000, dtype=np.uint64).astype(np.uint32)
    alt, nt = ref.ref_alt_policy(policy, bits, nb, b, t)
    got = np.array([o.alt_bucket(int(x), int(y)) for x, y in zip(b, t)], np.uint64)
    assert np.array_equal(got, alt)
    assert np.array_equal(np.array([o.alt_tag(int(y)) for y in t], np.uint32), nt)
    # the vectorised map agrees, and moving twice returns the tag home
    assert np.array_equal(o.alt_map()(b, t.astype(np.uint64)), alt)
    back = np.array([o.alt_bucket(int(x), int(y)) for x, y in zip(alt, nt)], np.uint64)
    assert np.array_equal(back, b)


@pytest.mark.parametrize("policy", [0, 1, 2])
def test_bucket_counts_match_reference(ref, policy):
    for cap in (1, 15, 16, 17, 1000, 1 << 20, 3_000_001):
        assert ref.num_buckets(cap, 16, policy) == int(ref.ref_host().ref_num_buckets_policy(policy, cap)), cap


@pytest.mark.parametrize("policy", POLICIES)
@pytest.mark.parametrize("evict", [0, 1])
def test_sequential_filter_with_policy(ref, policy, evict):
    o = ref.OracleFilter(bits=16, bucket_size=16, policy=evict, alt_policy=policy, capacity=50_000)
    if policy == 1:
        assert o.nb % 2 == 0
    keys = ref.splitmix64(77 + policy, int(0.95 * o.nb * 16))
    n, ok = o.insert(keys, out=True)
    assert n == ok.sum() and n == o.occupied()
    assert o.contains(keys[ok.astype(bool)]).all()
    slots = o.slots()
    i1, i2, fp = o.candidates(keys[ok.astype(bool)])
    errs = ref.check_invariants(slots, o.alt_map(), i1, i2, fp, norm=o.pure_tag)
    assert not errs, errs
    stored = keys[ok.astype(bool)]
    nd, out = o.delete(stored[: len(stored) // 2])
    assert nd == len(stored) // 2 and out.all()
    assert o.contains(stored[len(stored) // 2:]).all()
    assert o.occupied() == n - nd
