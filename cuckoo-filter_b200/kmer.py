"""k-mer sets on disk: the binary format the reference's k-mer benchmark reads.

The format (reference ``src/kmc_to_binary.cpp:1-7`` writes it,
``benchmark/kmer_benchmark.cu:26-46`` reads it) is one little-endian
``uint64`` count N followed by N little-endian ``uint64`` k-mers.  Each k-mer
(k <= 32) is 2-bit encoded, most significant base first, with A=0 C=1 G=2 T=3
(``kmc_to_binary.cpp:13-41``); a k-mer holding any other letter is not
encodable and is skipped by the converter.

``read_kmer_file`` raises, as the reference's loader does, when the file cannot
be opened, the count is missing or zero, or fewer than N k-mers follow.
"""
from __future__ import annotations

import os

import numpy as np

_CODE = {"A": 0, "C": 1, "G": 2, "T": 3, "a": 0, "c": 1, "g": 2, "t": 3}
NOT_ENCODABLE = (1 << 64) - 1  # kmc_to_binary.cpp's marker for a k-mer with another letter


def encode_kmer(kmer: str) -> int:
    """2-bit MSB-first encoding of one k-mer (``encodeKmer``), or
    ``NOT_ENCODABLE`` when it holds a letter other than A, C, G, T."""
    v = 0
    for c in kmer:
        b = _CODE.get(c)
        if b is None:
            return NOT_ENCODABLE
        v = (v << 2) | b
    return v & NOT_ENCODABLE


def canonical(code: int, k: int) -> int:
    """min(k-mer, its reverse complement), both 2-bit MSB-first."""
    rc = 0
    x = code
    for _ in range(k):
        rc = (rc << 2) | (3 - (x & 3))
        x >>= 2
    return min(code, rc)


def write_kmer_file(path: str | os.PathLike, kmers) -> int:
    """Write `kmers` (any integer array) in the binary format; returns N."""
    a = np.ascontiguousarray(np.asarray(kmers, dtype=np.uint64))
    with open(path, "wb") as f:
        f.write(np.uint64(a.size).astype("<u8").tobytes())
        f.write(a.astype("<u8", copy=False).tobytes())
    return int(a.size)


def read_kmer_file(path: str | os.PathLike) -> np.ndarray:
    """The k-mers of a binary k-mer file as a uint64 array."""
    try:
        f = open(path, "rb")
    except OSError as e:
        raise RuntimeError(f"Failed to open k-mer file: {path}") from e
    with f:
        head = f.read(8)
        if len(head) != 8:
            raise RuntimeError(f"Failed to read k-mer count from: {path}")
        n = int(np.frombuffer(head, dtype="<u8")[0])
        if n == 0:
            raise RuntimeError(f"Failed to read k-mer count from: {path}")
        body = f.read(8 * n)
        if len(body) != 8 * n:
            raise RuntimeError(f"Failed to read k-mers from: {path}")
    return np.frombuffer(body, dtype="<u8").astype(np.uint64)
