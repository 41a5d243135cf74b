"""Generate golden hashing vectors from the reference's own compiled code.

Runs where the reference sources exist (they are compiled by ``oracle/Makefile``
into ``oracle/_ref/libref_host.so`` from the reference's
``include/bucket_policies.cuh`` and ``include/hashutil.cuh``).  Writes
``tests/golden/candidates.npz``: for each configuration, the keys and the
reference's ``XorAltBucketPolicy::getCandidateBuckets`` output (i1, i2, fp)
plus raw ``xxhash64`` values of the keys and of every 8/16-bit tag.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

# (key_bytes, bits, bucket_size, capacity)
CASES = [
    (8, 16, 16, 1 << 20),       # small filter, 2^16 buckets
    (8, 8, 16, 1 << 31),        # large 8/16 filter, 2^27 buckets
    (8, 16, 16, 1 << 31),       # large 16/16 filter, 2^27 buckets
    (8, 32, 8, 1 << 31),        # large 32/8 filter, 2^28 buckets
    (8, 16, 16, (1 << 37)),     # 2^33 buckets: i2 reaches above 2^32
    (4, 16, 16, 10000),         # the reference unit-test configuration
    (4, 8, 32, 123457),
    (4, 32, 4, 999),
    (8, 16, 4, 1 << 12),
    (8, 8, 64, 1 << 26),
]

EDGE = [0, 1, 2, 3, 42, 100, 255, 256, 65535, 65536, (1 << 31), (1 << 32) - 1, 1 << 32, (1 << 32) + 1,
        1 << 63, (1 << 64) - 2, (1 << 64) - 1]


def fp_zero_keys(key_bytes: int, bits: int, count: int) -> list[int]:
    """Keys whose masked fingerprint is 0 (mapped to 1 by the policy)."""
    L = oracle.ref_host()
    cand = oracle.splitmix64(99, 400_000)
    if key_bytes == 4:
        cand = cand.astype(np.uint32)
    out = []
    mask = (1 << bits) - 1
    for k in cand:
        b = np.array([k]).view(np.uint8)[:key_bytes].copy()
        h = int(L.ref_xxhash64(b.ctypes.data, key_bytes))
        if ((h >> 32) & mask) == 0:
            out.append(int(k))
            if len(out) == count:
                break
    return out


def main() -> None:
    oracle.build()
    L = oracle.ref_host()
    if L is None:
        raise SystemExit("reference shim not built (needs the reference sources)")
    data = {}
    for ci, (kb, bits, bs, cap) in enumerate(CASES):
        nb = int(L.ref_num_buckets(cap, bs))
        rnd = oracle.splitmix64(1000 + ci, 1024)
        edge = [k for k in EDGE if k < (1 << (8 * kb))]
        zero = fp_zero_keys(kb, bits, 4) if bits <= 16 else []
        dt = np.uint64 if kb == 8 else np.uint32
        keys = np.concatenate([np.array(edge + zero, dtype=np.uint64).astype(dt), rnd.astype(dt)])
        i1, i2, fp = oracle.ref_candidates(kb, bits, bs, nb, keys)
        kh = np.array([L.ref_xxhash64(np.array([k], dtype=dt).ctypes.data, kb) for k in keys], dtype=np.uint64)
        pre = f"c{ci}_"
        data[pre + "meta"] = np.array([kb, bits, bs, cap, nb], dtype=np.uint64)
        data[pre + "keys"] = keys
        data[pre + "hash"] = kh
        data[pre + "i1"] = i1
        data[pre + "i2"] = i2
        data[pre + "fp"] = fp
    for nbytes in (1, 2):
        # every 8-bit tag; every 13th 16-bit tag plus the top of the range
        tags = np.arange(1 << (8 * nbytes), dtype=np.uint32)
        if nbytes == 2:
            tags = np.concatenate([tags[::13], tags[-16:]])
        data[f"tag{8 * nbytes}"] = tags
        data[f"taghash{8 * nbytes}"] = np.array(
            [L.ref_xxhash64(np.array([t], dtype=np.uint32).ctypes.data, nbytes) for t in tags], dtype=np.uint64)
    t32 = oracle.splitmix64(5, 1024).astype(np.uint32)
    data["tag32"] = t32
    data["taghash32"] = np.array([L.ref_xxhash64(np.array([t]).astype(np.uint32).ctypes.data, 4) for t in t32],
                                 dtype=np.uint64)
    data["num_buckets"] = np.array([[c, bs, L.ref_num_buckets(c, bs)] for c in
                                    (1, 2, 15, 16, 17, 1000, 10000, 996147, 1 << 20, (1 << 20) + 1, 1 << 31,
                                     (1 << 31) - 1, 3 << 29)
                                    for bs in (2, 4, 8, 16, 32, 64)], dtype=np.uint64)
    out = os.path.join(HERE, "candidates.npz")
    np.savez_compressed(out, **data)
    print(out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
