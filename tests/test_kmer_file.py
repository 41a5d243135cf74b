"""On-disk k-mer sets (cuckoo-filter_b200/kmer.py): the reference's binary
format (u64 count, then that many u64 2-bit MSB-first k-mers,
src/kmc_to_binary.cpp and benchmark/kmer_benchmark.cu:26-46)."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def km(cfb):
    import cuckoo_b200.kmer as k

    return k


def test_encoding_is_two_bit_msb_first(km):
    assert km.encode_kmer("A") == 0 and km.encode_kmer("T") == 3
    assert km.encode_kmer("ACGT") == 0b00011011
    assert km.encode_kmer("acgt") == km.encode_kmer("ACGT")
    assert km.encode_kmer("ACNT") == km.NOT_ENCODABLE
    assert km.encode_kmer("T" * 32) == (1 << 64) - 1  # 32 T's fill all 64 bits
    # canonical = min(forward, reverse complement)
    assert km.canonical(km.encode_kmer("AAAC"), 4) == km.encode_kmer("AAAC")
    assert km.canonical(km.encode_kmer("GTTT"), 4) == km.encode_kmer("AAAC")


def test_bench_canonical_kmers_agree_with_the_string_encoding(km):
    import torch

    import bench

    rng = np.random.default_rng(5)
    b = rng.integers(0, 4, 120).astype(np.uint8)
    s = "".join("ACGT"[x] for x in b)
    got = bench.canonical_kmers(torch.from_numpy(b), k=31).numpy().view(np.uint64)
    want = [km.canonical(km.encode_kmer(s[i:i + 31]), 31) for i in range(len(s) - 30)]
    assert got.tolist() == want


def test_round_trip_and_layout(km, tmp_path):
    kmers = np.array([0, 1, 2**62 + 5, 2**64 - 2], np.uint64)
    p = tmp_path / "k.bin"
    assert km.write_kmer_file(p, kmers) == 4
    raw = p.read_bytes()
    assert len(raw) == 8 * 5 and int.from_bytes(raw[:8], "little") == 4
    assert int.from_bytes(raw[8 * 3:8 * 4], "little") == 2**62 + 5
    got = km.read_kmer_file(p)
    assert got.dtype == np.uint64 and np.array_equal(got, kmers)


def test_errors_like_the_reference_loader(km, tmp_path):
    with pytest.raises(RuntimeError, match="Failed to open"):
        km.read_kmer_file(tmp_path / "missing.bin")
    empty = tmp_path / "zero.bin"
    empty.write_bytes((0).to_bytes(8, "little"))
    with pytest.raises(RuntimeError, match="count"):
        km.read_kmer_file(empty)
    short = tmp_path / "short.bin"
    short.write_bytes((3).to_bytes(8, "little") + (7).to_bytes(8, "little"))
    with pytest.raises(RuntimeError, match="Failed to read k-mers"):
        km.read_kmer_file(short)
    noc = tmp_path / "nocount.bin"
    noc.write_bytes(b"\x01\x02")
    with pytest.raises(RuntimeError, match="count"):
        km.read_kmer_file(noc)


@pytest.mark.gpu
def test_a_kmer_file_fills_a_filter(cfb, km, tmp_path):
    """k-mers of synthetic DNA written to a file, read back, inserted to 0.95
    load: every one is found, and the counters match the set size."""
    import torch

    import bench

    dna = bench.markov_dna(1 << 16, 64, seed=9, device=torch.device("cpu"))
    kmers = np.unique(bench.canonical_kmers(dna, k=31).numpy().view(np.uint64))
    p = tmp_path / "set.bin"
    km.write_kmer_file(p, kmers)
    got = km.read_kmer_file(p)
    cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=16, bucketSize=16, evictionPolicy=cfb.EvictionPolicy.BFS)
    f = cfb.CuckooFilter(cfg, int(got.size / 0.95))
    d = torch.from_numpy(got.view(np.int64)).cuda()
    occ = f.insertMany(d)
    assert occ == got.size and f.stats()["failed"] == 0
    out = torch.zeros(got.size, dtype=torch.bool, device="cuda")
    f.containsMany(d, out)
    assert bool(out.all())
    f.close()
