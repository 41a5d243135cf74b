"""Host logic of bench.py: key generators, disjointness and the parity check's hashing and digests (CPU only)."""
from __future__ import annotations

import numpy as np
import torch

import bench


def test_torch_splitmix64_matches_oracle(orc):
    for seed, first, n in ((3, 0, 1000), (4, 12345, 777), (1, 0, 1 << 16)):
        t = torch.empty(n, dtype=torch.int64)
        bench.splitmix64_torch(seed, first, n, t, chunk=4096)
        assert np.array_equal(t.numpy().view(np.uint64), orc.splitmix64(seed, n, first))


def test_negative_collisions_exact():
    # seed_neg = seed_pos + 5*gamma: negative j equals positive j + 5
    sp = 3
    sn = (sp + 5 * bench.G) % bench.U64
    bad = bench.negative_collisions(sp, 100, sn, 200)
    assert bad == list(range(0, 95))
    assert bench.collides(sp, 100, sn, 94) and not bench.collides(sp, 100, sn, 95)
    # the default seeds of the workloads do not collide
    for w in bench.WORKLOADS.values():
        n_fill = int(w["fill"] * w["capacity"])
        assert bench.negative_collisions(w["seed_fill"], n_fill, w["seed_neg"], w["n_neg"]) == []


def test_negative_collisions_against_brute_force(orc):
    sp, sn = 11, (11 + 1000 * bench.G) % bench.U64
    pos = orc.splitmix64(sp, 3000)
    neg = orc.splitmix64(sn, 3000)
    brute = [j for j in range(3000) if neg[j] in set(pos.tolist())]
    assert bench.negative_collisions(sp, 3000, sn, 3000) == brute


def test_small_workload_inputs_cpu():
    w = dict(bench.WORKLOADS["small"])
    fill, query, dele, n_coll = bench.make_inputs(w, torch.device("cpu"))
    assert n_coll == 0
    assert fill.numel() == int(0.95 * (1 << 20)) == 996147
    assert query.numel() == 2 * 996147 and dele.numel() == 996147 // 2
    assert torch.unique(fill).numel() == fill.numel()
    pos = set(fill.tolist())
    q = query.tolist()
    assert sum(1 for x in q if x in pos) == 996147
    assert all(x in pos for x in dele.tolist())


def test_positive_sample_without_replacement():
    w = dict(bench.WORKLOADS["small"], capacity=1 << 16, n_pos=20000, n_neg=20000, n_del=5000, seed_sample=9)
    fill, query, dele, _ = bench.make_inputs(w, torch.device("cpu"))
    pos = set(fill.tolist())
    qp = [x for x in query.tolist() if x in pos]
    assert len(qp) == 20000 == len(set(qp))


def test_segmented_splitmix64_matches_oracle(orc):
    """The batched form's key generator: segment i is splitmix64(seed_i) from output first_i."""
    import numpy as np
    import torch

    import bench

    seeds = np.array([0, 7, 4095, 1 << 40], np.int64)
    counts = np.array([5, 0, 17, 3], np.int64)
    first = np.array([0, 0, 2, 1], np.int64)
    got = bench.splitmix64_segments(seeds, counts, first, torch.device("cpu")).numpy().view(np.uint64)
    want = np.concatenate([orc.splitmix64(int(s), int(c) + int(f))[int(f):] for s, c, f in zip(seeds, counts, first)])
    assert np.array_equal(got, want)


def test_canonical_kmers_match_a_direct_encoding():
    """2-bit MSB-first encoding (A0 C1 G2 T3), canonical = min(forward, reverse complement)."""
    import numpy as np
    import torch

    import bench

    rng = np.random.default_rng(0)
    b = rng.integers(0, 4, 200).astype(np.uint8)
    got = bench.canonical_kmers(torch.from_numpy(b), k=31).numpy()
    for i in (0, 1, 77, 169):
        w = b[i:i + 31]
        fwd = sum(int(x) << (2 * (30 - j)) for j, x in enumerate(w))
        rc = sum(int(3 - x) << (2 * (30 - j)) for j, x in enumerate(w[::-1]))
        assert got[i] == min(fwd, rc)
    # a window and its reverse complement share the canonical k-mer
    rcs = (3 - b[::-1]).copy()
    got_rc = bench.canonical_kmers(torch.from_numpy(rcs), k=31).numpy()
    assert set(got.tolist()) == set(got_rc.tolist())


def test_markov_dna_and_mutation_cpu():
    import torch

    import bench

    dna = bench.markov_dna(1 << 12, 16, seed=1, device=torch.device("cpu"))
    assert dna.numel() == 4096 and int(dna.max()) <= 3
    m = bench.mutate(dna, 0.01, seed=2)
    diff = (m != dna).float().mean().item()
    assert 0.0 < diff < 0.03


# ------------------------------------- the parity check's hashing and digests


def test_parity_hashing_matches_reference_golden(golden):
    """bench.py's torch restatement of xxHash64 and XorAltBucketPolicy against the
    vectors generated from the reference's own hashutil.cuh / bucket_policies.cuh."""
    for i in range(10):
        kb, bits, _bs, _cap, nb = (int(x) for x in golden[f"c{i}_meta"])
        keys = golden[f"c{i}_keys"]
        kt = torch.from_numpy(keys.view(np.int64) if keys.dtype == np.uint64 else keys.astype(np.int64))
        h = bench.xxh64_torch(kt, kb).numpy().view(np.uint64)
        assert np.array_equal(h, golden[f"c{i}_hash"]), i
        i1, i2, fp = bench.candidates_torch(kt, kb, bits, nb, bench.tag_hash_table(bits, "cpu") if bits <= 16 else None)
        assert np.array_equal(i1.numpy().view(np.uint64), golden[f"c{i}_i1"]), i
        assert np.array_equal(i2.numpy().view(np.uint64), golden[f"c{i}_i2"]), i
        assert np.array_equal(fp.numpy().astype(np.uint32), golden[f"c{i}_fp"]), i
    for b in (8, 16, 32):
        t = torch.from_numpy(golden[f"tag{b}"].astype(np.int64))
        assert np.array_equal(bench.xxh64_torch(t, b // 8).numpy().view(np.uint64), golden[f"taghash{b}"]), b


def _oracle_filled(orc, bits, seed=5):
    o = orc.OracleFilter(key_bytes=8, bits=bits, bucket_size=16, policy=orc.POLICY_BFS, capacity=1 << 16)
    keys = orc.splitmix64(seed, int(0.95 * (1 << 16)))
    _, ok = o.insert(keys, out=True)
    return o, keys, ok.astype(bool)


def test_digests_agree_on_an_oracle_table(orc):
    for bits in (8, 16):
        o, keys, ok = _oracle_filled(orc, bits)
        kt = torch.from_numpy(keys.view(np.int64))
        stored = bench.key_digest(kt, bits, o.nb, valid=torch.from_numpy(ok), chunk=1 << 12)
        table = bench.table_digest(torch.from_numpy(o.table), bits, 16, o.nb, chunk_slots=1 << 12)
        assert stored == table and stored[0] == o.occupied() == int(ok.sum()), bits
        # deleting a subset removes exactly its entries from the multiset
        gone = keys[ok][:5000]
        n, _ = o.delete(gone)
        assert n == 5000
        after = bench.table_digest(torch.from_numpy(o.table), bits, 16, o.nb)
        assert after == bench.digest_sub(stored, bench.key_digest(torch.from_numpy(gone.view(np.int64)), bits, o.nb))


def test_digest_catches_a_planted_mistake_in_the_oracle_table(orc):
    o, keys, ok = _oracle_filled(orc, 16)
    want = bench.key_digest(torch.from_numpy(keys.view(np.int64)), 16, o.nb, valid=torch.from_numpy(ok))
    slots = o.slots()
    b, s = np.argwhere(slots != 0)[123]
    # a tag moved to a bucket that is neither of its key's candidates
    moved = o.table.copy()
    mv = moved.view(np.uint16).reshape(o.nb, 16)
    free = np.argwhere(mv[(b + 1) % o.nb] == 0)
    if len(free):
        mv[(b + 1) % o.nb, free[0][0]] = mv[b, s]
        mv[b, s] = 0
        assert bench.table_digest(torch.from_numpy(moved), 16, 16, o.nb) != want
    # a tag changed in place
    changed = o.table.copy()
    changed.view(np.uint16).reshape(o.nb, 16)[b, s] ^= 1
    assert bench.table_digest(torch.from_numpy(changed), 16, 16, o.nb) != want
    # a tag dropped
    dropped = o.table.copy()
    dropped.view(np.uint16).reshape(o.nb, 16)[b, s] = 0
    assert bench.table_digest(torch.from_numpy(dropped), 16, 16, o.nb) != want
