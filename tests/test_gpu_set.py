"""Filter sets (the batched form): many filters, uneven batches, one launch.

* lookups on identical table images equal the oracle's, filter by filter, for
  every launch shape the autotuner can pick (blocks x keys per thread x probe
  widths), and inside a captured CUDA graph replayed with new keys;
* batched inserts keep every per-filter invariant (no false negatives, the
  (bucket pair, tag) multiset of each table equals its stored keys', counters
  equal the images);
* batched deletes remove one copy per key;
* a work item naming a filter outside the set is reported, its keys skipped;
* the set agrees with a loop of single-filter calls (the reference's usage).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from test_gpu_parity import alt_fn, dev, host_u8  # noqa: E402


def make_set(cfb, orc, bits, bs, caps, policy=0):
    cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=bits, bucketSize=bs, evictionPolicy=cfb.EvictionPolicy(policy))
    s = cfb.CuckooFilterSet(cfg, caps)
    oracles = [orc.OracleFilter(key_bytes=8, bits=bits, bucket_size=bs, policy=policy, capacity=int(c),
                                mode=orc.MODE_CONSERVING) for c in caps]
    for i, o in enumerate(oracles):
        assert s.num_buckets[i] == o.nb
    return s, oracles


def work_list(batches):
    """Concatenated keys, offsets and filter ids of [(filter, keys), ...]."""
    keys = np.concatenate([k for _, k in batches]) if batches else np.zeros(0, np.uint64)
    offs = np.zeros(len(batches) + 1, np.int64)
    offs[1:] = np.cumsum([len(k) for _, k in batches])
    filt = np.array([f for f, _ in batches], np.int32)
    return dev(keys), torch.from_numpy(offs).cuda(), torch.from_numpy(filt).cuda(), keys


def uneven_caps(n, lo=10, hi=16, seed=0):
    rng = np.random.default_rng(seed)
    return np.exp2(rng.uniform(lo, hi, n)).astype(np.uint64)


GEOMS = [(16, 16), (8, 16), (32, 8)]


@pytest.mark.parametrize("bits,bs", GEOMS)
def test_set_lookups_match_oracle_for_every_launch_shape(cfb, orc, bits, bs):
    caps = uneven_caps(23, seed=bits)
    s, oracles = make_set(cfb, orc, bits, bs, caps)
    batches = []
    for i, o in enumerate(oracles):
        keys = orc.splitmix64(100 + i, int(0.9 * o.nb * o.bucket_size))
        o.insert(keys)
        s.load_table(i, torch.from_numpy(o.table))
        neg = orc.splitmix64(5000 + i, 700)
        q = np.concatenate([keys[: 900], neg])
        # uneven items, one filter split over two items, empty items mixed in
        batches += [(i, q[:500]), (i, np.zeros(0, np.uint64)), (i, q[500:])]
    d_keys, d_offs, d_filt, h_keys = work_list(batches)
    want = np.concatenate([o.contains(q) for (i, q), o in
                           zip(batches, [oracles[i] for i, _ in batches])]) if batches else None
    widths = [1, 4, 8] if bits * bs // 8 == 32 else [1, 2, 4]
    for block in (128, 256, 512):
        for kpt in (1, 2, 4, 8):
            for w in widths:
                s.set_launch(cfb.SET_CONTAINS, block, kpt, w)
                out = torch.full((len(h_keys),), 7, dtype=torch.uint8, device="cuda")
                s.contains_async(d_keys, d_offs, d_filt, out)
                s.sync()
                assert np.array_equal(host_u8(out), want), (block, kpt, w)


def test_set_inserts_keep_every_filter_invariant(cfb, orc):
    caps = uneven_caps(64, lo=10, hi=18, seed=3)
    s, oracles = make_set(cfb, orc, 16, 16, caps, policy=0)
    rng = np.random.default_rng(4)
    batches, per_filter = [], []
    for i, o in enumerate(oracles):
        n = int(min(0.9 * o.nb * 16, rng.lognormal(np.log(2000), 1.5)))
        keys = orc.splitmix64(300 + i, n)
        per_filter.append(keys)
        half = n // 2
        batches += [(i, keys[:half]), (i, keys[half:])]
    rng.shuffle(batches)  # items of one filter need not be adjacent
    d_keys, d_offs, d_filt, h_keys = work_list(batches)
    ok = torch.zeros(len(h_keys), dtype=torch.uint8, device="cuda")
    s.insert_async(d_keys, d_offs, d_filt, ok)
    s.sync()
    ok_h = host_u8(ok).astype(bool)
    occ = s.occupied()
    for i, o in enumerate(oracles):
        st = s.stats(i)
        img = s.table_image(i).numpy()
        slots = img.view(np.uint16).reshape(o.nb, 16)
        assert st["lost"] == 0 and st["failed"] == 0, (i, st)
        assert int(occ[i]) == int((slots != 0).sum()) == len(per_filter[i]), i
        i1, i2, fp = o.candidates(per_filter[i])
        errs = orc.check_invariants(slots, alt_fn(orc, o), i1, i2, fp)
        assert not errs, (i, errs)
    assert ok_h.all()
    out = torch.zeros(len(h_keys), dtype=torch.uint8, device="cuda")
    s.contains_async(d_keys, d_offs, d_filt, out)
    s.sync()
    assert host_u8(out).all(), "false negative"


def test_set_deletes_remove_one_copy_per_key(cfb, orc):
    caps = uneven_caps(16, seed=7)
    s, oracles = make_set(cfb, orc, 16, 16, caps)
    batches = []
    for i, o in enumerate(oracles):
        keys = orc.splitmix64(400 + i, int(0.8 * o.nb * 16))
        o.insert(keys)
        s.load_table(i, torch.from_numpy(o.table))
        batches.append((i, keys))
    d_keys, d_offs, d_filt, h_keys = work_list(batches)
    # counters follow the loaded images
    occ0 = np.array([o.occupied() for o in oracles])
    s.clear()
    for i, o in enumerate(oracles):
        s.load_table(i, torch.from_numpy(o.table))
    dels = [(i, k[: len(k) // 2]) for i, k in batches]
    dk, do, df, dh = work_list(dels)
    out = torch.zeros(len(dh), dtype=torch.uint8, device="cuda")
    s.delete_async(dk, do, df, out)
    s.sync()
    assert host_u8(out).all(), "a stored key was not deleted"
    for i, o in enumerate(oracles):
        o.delete(dels[i][1])
        img = s.table_image(i).numpy()
        assert int((img.view(np.uint16) != 0).sum()) == o.occupied() == occ0[i] - len(dels[i][1])
        assert s.stats(i)["removed"] == len(dels[i][1])
    # the rest is still there
    rest = [(i, k[len(k) // 2:]) for i, k in batches]
    rk, ro, rf, rh = work_list(rest)
    out = torch.zeros(len(rh), dtype=torch.uint8, device="cuda")
    s.contains_async(rk, ro, rf, out)
    s.sync()
    assert host_u8(out).all()


def test_set_lookup_graph_replay(cfb, orc):
    caps = uneven_caps(40, seed=9)
    s, oracles = make_set(cfb, orc, 16, 16, caps)
    batches = []
    for i, o in enumerate(oracles):
        keys = orc.splitmix64(500 + i, int(0.85 * o.nb * 16))
        o.insert(keys)
        s.load_table(i, torch.from_numpy(o.table))
        batches.append((i, np.concatenate([keys[:300], orc.splitmix64(900 + i, 300)])))
    d_keys, d_offs, d_filt, h_keys = work_list(batches)
    out = torch.zeros(len(h_keys), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    s.contains_async(d_keys, d_offs, d_filt, out, stream=stream)  # warm-up outside capture
    s.sync(stream=stream)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        s.contains_async(d_keys, d_offs, d_filt, out, stream=stream)
    for rnd in range(3):
        # new keys in the same buffer, same work list
        batches2 = [(i, np.concatenate([orc.splitmix64(500 + i, int(0.85 * o.nb * 16))[rnd * 50: rnd * 50 + 300],
                                        orc.splitmix64(7000 + 10 * i + rnd, 300)])) for i, o in enumerate(oracles)]
        h2 = np.concatenate([k for _, k in batches2])
        d_keys.copy_(torch.from_numpy(h2.view(np.int64)))
        out.fill_(9)
        g.replay()
        torch.cuda.synchronize()
        want = np.concatenate([oracles[i].contains(k) for i, k in batches2])
        assert np.array_equal(host_u8(out), want), rnd
    del g


def test_set_rejects_foreign_filter_ids(cfb, orc):
    s, oracles = make_set(cfb, orc, 16, 16, [1 << 12, 1 << 12])
    keys = orc.splitmix64(1, 1000)
    d_keys, d_offs, d_filt, _ = work_list([(0, keys[:500]), (5, keys[500:])])
    out = torch.zeros(1000, dtype=torch.uint8, device="cuda")
    s.insert_async(d_keys, d_offs, d_filt, out)
    with pytest.raises(cfb.CuckooError) as e:
        s.sync()
    assert e.value.status == -1
    assert host_u8(out)[:500].all() and not host_u8(out)[500:].any()
    assert s.occupied().tolist() == [500, 0]
    s.sync()  # the error was reported once


def test_set_autotune_and_agreement_with_single_filters(cfb, orc):
    caps = uneven_caps(32, lo=12, hi=18, seed=11)
    s, oracles = make_set(cfb, orc, 16, 16, caps)
    batches = []
    singles = []
    cfg = s.config
    for i, o in enumerate(oracles):
        keys = orc.splitmix64(600 + i, int(0.9 * o.nb * 16))
        f = cfb.CuckooFilter(cfg, int(caps[i]))
        f.insertMany(dev(keys))
        s.load_table(i, f.table_image())
        singles.append(f)
        batches.append((i, np.concatenate([keys[::2], orc.splitmix64(8000 + i, 2000)])))
    d_keys, d_offs, d_filt, h_keys = work_list(batches)
    out = torch.zeros(len(h_keys), dtype=torch.uint8, device="cuda")
    best = s.autotune(cfb.SET_CONTAINS, d_keys, d_offs, d_filt, out)
    assert best > 0
    block, kpt, width = s.get_launch(cfb.SET_CONTAINS)
    assert block in (128, 256, 512) and kpt in (1, 2, 4, 8) and width in (1, 4, 8)
    s.contains_async(d_keys, d_offs, d_filt, out)
    s.sync()
    want = np.concatenate([host_u8(f.containsMany(dev(k))) for f, (_, k) in zip(singles, batches)])
    assert np.array_equal(host_u8(out), want)
    # tuning inserts leaves the set empty
    s.autotune(cfb.SET_INSERT, d_keys, d_offs, d_filt)
    assert int(s.occupied().sum()) == 0
