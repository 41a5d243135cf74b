"""Test oracle for the cuckoo filter batch path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline / reference legs of ``bench.py``.  The CUDA library never
imports it.

Three native pieces are wrapped here:

* ``_build/libcf_oracle.so`` -- the C restatement (``cf_oracle.c``) of the
  reference's hashing, bucket policy and sequential insert/lookup/delete
  (reference ``include/CuckooFilter.cuh:805-1116``), plus a multithreaded port
  used as the CPU baseline.
* ``_ref/libref_host.so`` -- the reference's own ``XorAltBucketPolicy`` and
  ``xxhash64`` compiled from its headers (pins the restatement's hashing).
* ``_ref/libref_gpu.so`` -- the reference's own CUDA kernels (run only where a GPU is present).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libcf_oracle.so")
REF_HOST_SO = os.path.join(HERE, "_ref", "libref_host.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libref_gpu.so")

POLICY_BFS, POLICY_DFS = 0, 1
ALT_XOR, ALT_ADDSUB, ALT_OFFSET = 0, 1, 2
MODE_REFERENCE, MODE_CONSERVING = 0, 1
STAT_NAMES = ("primary", "secondary", "evicted_inserts", "evictions", "failed")


class Params(C.Structure):
    _fields_ = [
        ("key_bytes", C.c_uint32),
        ("bits", C.c_uint32),
        ("bucket_size", C.c_uint32),
        ("word_bytes", C.c_uint32),
        ("policy", C.c_uint32),
        ("max_evictions", C.c_uint32),
        ("num_buckets", C.c_uint64),
        ("alt_policy", C.c_uint32),
    ]


_lib = None


def build() -> None:
    """Compile the oracle (and the reference shims when the sources exist)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        vp, sz, u64, u32 = C.c_void_p, C.c_size_t, C.c_uint64, C.c_uint32
        P = C.POINTER(Params)
        L.cfo_xxhash64.argtypes = [vp, sz]
        L.cfo_xxhash64.restype = u64
        L.cfo_num_buckets.argtypes = [u64, u32]
        L.cfo_num_buckets.restype = u64
        L.cfo_num_buckets_policy.argtypes = [u64, u32, u32]
        L.cfo_num_buckets_policy.restype = u64
        L.cfo_alt_tag.argtypes = [P, u32]
        L.cfo_alt_tag.restype = u32
        L.cfo_alt_bucket.argtypes = [P, u64, u32]
        L.cfo_alt_bucket.restype = u64
        L.cfo_candidates.argtypes = [P, vp, sz, vp, vp, vp]
        L.cfo_candidates.restype = None
        L.cfo_insert_seq.argtypes = [P, vp, vp, sz, vp, C.c_int, vp]
        L.cfo_insert_seq.restype = sz
        L.cfo_delete_seq.argtypes = [P, vp, vp, sz, vp]
        L.cfo_delete_seq.restype = sz
        L.cfo_count_occupied.argtypes = [P, vp]
        L.cfo_count_occupied.restype = sz
        L.cfo_probe_count.argtypes = [P, vp, vp, sz]
        L.cfo_probe_count.restype = u64
        for name in ("cfo_insert_mt", "cfo_contains_mt", "cfo_delete_mt"):
            f = getattr(L, name)
            f.argtypes = [P, vp, vp, sz, vp, C.c_int]
            f.restype = sz
        L.cfo_splitmix64.argtypes = [u64, u64, sz, vp]
        L.cfo_splitmix64.restype = None
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def splitmix64(seed: int, n: int, first: int = 0) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    lib().cfo_splitmix64(seed, first, n, _ptr(out))
    return out


def xxhash64(value: int, nbytes: int) -> int:
    b = np.array([value], dtype=np.uint64).view(np.uint8)[:nbytes].copy()
    return int(lib().cfo_xxhash64(_ptr(b), nbytes))


def num_buckets(capacity: int, bucket_size: int, alt_policy: int = ALT_XOR) -> int:
    return int(lib().cfo_num_buckets_policy(capacity, bucket_size, alt_policy))


@dataclass
class OracleFilter:
    """Sequential host filter with the reference's layout and semantics."""

    key_bytes: int = 8
    bits: int = 16
    bucket_size: int = 16
    word_bytes: int = 8
    policy: int = POLICY_DFS
    max_evictions: int = 500
    capacity: int = 1 << 20
    mode: int = MODE_CONSERVING
    alt_policy: int = ALT_XOR

    def __post_init__(self):
        self.nb = num_buckets(self.capacity, self.bucket_size, self.alt_policy)
        self.p = Params(self.key_bytes, self.bits, self.bucket_size, self.word_bytes, self.policy,
                        self.max_evictions, self.nb, self.alt_policy)
        self.bucket_bytes = self.bucket_size * self.bits // 8
        self.table = np.zeros(self.nb * self.bucket_bytes, dtype=np.uint8)
        self.stats = np.zeros(len(STAT_NAMES), dtype=np.uint64)

    @property
    def key_dtype(self):
        return np.uint64 if self.key_bytes == 8 else np.uint32

    def _keys(self, keys) -> np.ndarray:
        return np.ascontiguousarray(keys, dtype=self.key_dtype)

    def candidates(self, keys):
        k = self._keys(keys)
        i1 = np.empty(len(k), np.uint64)
        i2 = np.empty(len(k), np.uint64)
        fp = np.empty(len(k), np.uint32)
        lib().cfo_candidates(C.byref(self.p), _ptr(k), len(k), _ptr(i1), _ptr(i2), _ptr(fp))
        return i1, i2, fp

    def alt_bucket(self, bucket: int, tag: int) -> int:
        return int(lib().cfo_alt_bucket(C.byref(self.p), bucket, tag))

    def alt_tag(self, tag: int) -> int:
        """The tag as stored in its alternate bucket (Offset policy: choice bit flipped)."""
        return int(lib().cfo_alt_tag(C.byref(self.p), tag))

    def alt_map(self):
        """Vectorised (bucket, tag) -> alternate bucket for this filter's policy."""
        return alt_vectorized(self.bits, self.nb, self.alt_policy)

    def pure_tag(self, tags):
        """Tags without the Offset policy's choice bit (unchanged otherwise)."""
        t = np.asarray(tags).astype(np.uint64)
        if self.alt_policy == ALT_OFFSET:
            t = t & np.uint64((1 << (self.bits - 1)) - 1)
        return t

    def insert(self, keys, out: bool = False):
        k = self._keys(keys)
        o = np.empty(len(k), np.uint8) if out else None
        n = lib().cfo_insert_seq(C.byref(self.p), _ptr(self.table), _ptr(k), len(k), _ptr(o), self.mode,
                                 _ptr(self.stats))
        return (n, o) if out else n

    def contains(self, keys, threads: int = 1) -> np.ndarray:
        k = self._keys(keys)
        o = np.empty(len(k), np.uint8)
        lib().cfo_contains_mt(C.byref(self.p), _ptr(self.table), _ptr(k), len(k), _ptr(o), threads)
        return o

    def delete(self, keys):
        k = self._keys(keys)
        o = np.empty(len(k), np.uint8)
        n = lib().cfo_delete_seq(C.byref(self.p), _ptr(self.table), _ptr(k), len(k), _ptr(o))
        return n, o

    def occupied(self) -> int:
        return int(lib().cfo_count_occupied(C.byref(self.p), _ptr(self.table)))

    def probe_count(self, keys) -> int:
        k = self._keys(keys)
        return int(lib().cfo_probe_count(C.byref(self.p), _ptr(self.table), _ptr(k), len(k)))

    def slots(self) -> np.ndarray:
        """Table image as (num_buckets, bucket_size) tag array."""
        dt = {8: np.uint8, 16: np.uint16, 32: np.uint32}[self.bits]
        return self.table.view(dt).reshape(self.nb, self.bucket_size)


def check_invariants(slots: np.ndarray, alt_of, keys_i1, keys_i2, keys_fp, norm=None) -> list[str]:
    """Structural checks on a table image.

    ``slots`` is (nb, bs) tags; ``keys_*`` are the candidates of the keys that
    are supposed to be stored (one entry per successful insert).  Returns a list
    of violations (empty when the image is consistent):
      * every stored key's tag sits in one of its two buckets (no false negatives),
      * the multiset {(min(b, alt), max(b, alt), tag)} of stored entries equals the
        multiset of the inserted keys' {(min(i1,i2), max(i1,i2), fp)}.
    ``norm`` maps tags to the form compared (the Offset policy's tags without
    their choice bit); identity when None.
    """
    norm = norm or (lambda x: np.asarray(x).astype(np.uint64))
    errs = []
    b_idx, s_idx = np.nonzero(slots)
    tags = slots[b_idx, s_idx].astype(np.uint64)
    alts = alt_of(b_idx.astype(np.uint64), tags)
    lo = np.minimum(b_idx.astype(np.uint64), alts)
    hi = np.maximum(b_idx.astype(np.uint64), alts)
    table_set = np.stack([lo, hi, norm(tags)], axis=1)
    klo = np.minimum(keys_i1, keys_i2).astype(np.uint64)
    khi = np.maximum(keys_i1, keys_i2).astype(np.uint64)
    key_set = np.stack([klo, khi, norm(keys_fp)], axis=1)
    if len(table_set) != len(key_set):
        errs.append(f"entry count {len(table_set)} != stored keys {len(key_set)}")
    ts = table_set[np.lexsort(table_set.T[::-1])]
    ks = key_set[np.lexsort(key_set.T[::-1])]
    if len(ts) == len(ks) and not np.array_equal(ts, ks):
        errs.append("bucket-pair/tag multiset differs from the stored keys")
    return errs


def alt_vectorized(bits: int, nb: int, alt_policy: int = ALT_XOR):
    """Vectorised alternate-bucket map (per-tag hash lookup table for tags of
    up to 16 bits) for the XOR, AddSub and Offset policies."""
    ntags = 1 << min(bits, 16)
    if bits <= 16:
        tbl = np.array([xxhash64(t, bits // 8) for t in range(ntags)], dtype=np.uint64)

        def th(t):
            return tbl[np.asarray(t).astype(np.int64)]
    else:
        def th(t):
            return np.array([xxhash64(int(x), 4) for x in np.asarray(t)], dtype=np.uint64)

    nbu = np.uint64(nb)
    if alt_policy == ALT_ADDSUB:
        half = np.uint64(nb // 2)

        def f(b, t):
            b = np.asarray(b).astype(np.uint64)
            fh = th(t) % half
            return np.where(b < half, (b + fh) % half + half, (b - fh) % half)
    elif alt_policy == ALT_OFFSET:
        cb = np.uint64(1 << (bits - 1))

        def f(b, t):
            b = np.asarray(b).astype(np.uint64)
            t = np.asarray(t).astype(np.uint64)
            off = th(t & (cb - np.uint64(1))) % nbu
            off = np.where(off == 0, np.uint64(1), off)
            return np.where((t & cb) == 0, (b + off) % nbu, (b + nbu - off) % nbu)
    else:
        def f(b, t):
            return np.asarray(b).astype(np.uint64) ^ (th(t) & np.uint64(nb - 1))
    return f


# ------------------------------------------------------------- reference shims

_ref_host = None


def ref_host():
    """The reference's own hashing (compiled from its headers), or None."""
    global _ref_host
    if _ref_host is None and os.path.exists(REF_HOST_SO):
        L = C.CDLL(REF_HOST_SO)
        L.ref_candidates.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p, C.c_size_t,
                                     C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_candidates.restype = C.c_int
        L.ref_xxhash64.argtypes = [C.c_void_p, C.c_size_t]
        L.ref_xxhash64.restype = C.c_uint64
        L.ref_num_buckets.argtypes = [C.c_uint64, C.c_uint32]
        L.ref_num_buckets.restype = C.c_uint64
        L.ref_candidates_policy.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p,
                                            C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_candidates_policy.restype = C.c_int
        L.ref_alt_policy.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_size_t,
                                     C.c_void_p, C.c_void_p]
        L.ref_alt_policy.restype = C.c_int
        L.ref_num_buckets_policy.argtypes = [C.c_uint32, C.c_uint64]
        L.ref_num_buckets_policy.restype = C.c_uint64
        _ref_host = L
    return _ref_host


def ref_candidates(key_bytes, bits, bucket_size, nb, keys):
    L = ref_host()
    k = np.ascontiguousarray(keys, dtype=np.uint64 if key_bytes == 8 else np.uint32)
    i1 = np.empty(len(k), np.uint64)
    i2 = np.empty(len(k), np.uint64)
    fp = np.empty(len(k), np.uint32)
    rc = L.ref_candidates(key_bytes, bits, bucket_size, nb, _ptr(k), len(k), _ptr(i1), _ptr(i2), _ptr(fp))
    assert rc == 0
    return i1, i2, fp


# Configuration ids of oracle/ref_gpu.cu's kOps table.
REF_GPU_CONFIGS = {
    # (key_bytes, bits, bucket_size, policy, max_evictions): id
    (8, 16, 16, POLICY_BFS, 500): 0,
    (8, 16, 16, POLICY_DFS, 500): 1,
    (8, 8, 16, POLICY_BFS, 500): 2,
    (8, 8, 16, POLICY_DFS, 500): 3,
    (8, 32, 8, POLICY_BFS, 500): 4,
    (8, 32, 8, POLICY_DFS, 500): 5,
    (4, 16, 16, POLICY_DFS, 500): 6,
    (8, 16, 16, POLICY_DFS, 16): 7,
    (8, 16, 16, POLICY_BFS, 16): 8,
    (8, 32, 8, POLICY_DFS, 16): 9,
    (8, 32, 8, POLICY_BFS, 16): 10,
    # 32-bit WordType: (key_bytes, bits, bucket_size, policy, max_evictions, word_bytes)
    (8, 8, 16, POLICY_DFS, 500, 4): 11,
    (8, 8, 16, POLICY_BFS, 500, 4): 12,
    (8, 16, 16, POLICY_DFS, 500, 4): 13,
    (8, 16, 16, POLICY_BFS, 16, 4): 14,
    # other alternate-bucket policies: (..., word_bytes, alt_policy)
    (8, 16, 16, POLICY_BFS, 500, 8, ALT_ADDSUB): 15,
    (8, 16, 16, POLICY_DFS, 500, 8, ALT_ADDSUB): 16,
    (8, 16, 16, POLICY_BFS, 500, 8, ALT_OFFSET): 17,
    (8, 16, 16, POLICY_DFS, 500, 8, ALT_OFFSET): 18,
    (8, 16, 16, POLICY_DFS, 16, 8, ALT_OFFSET): 19,
    (8, 16, 16, POLICY_DFS, 16, 8, ALT_ADDSUB): 20,
}

_ref_gpu = None


def ref_gpu():
    """The reference's own CUDA kernels (needs a GPU), or None if not built."""
    global _ref_gpu
    if _ref_gpu is None and os.path.exists(REF_GPU_SO):
        L = C.CDLL(REF_GPU_SO)
        vp, sz = C.c_void_p, C.c_size_t
        L.refg_create.argtypes = [C.c_int, sz]
        L.refg_create.restype = vp
        L.refg_destroy.argtypes = [C.c_int, vp]
        L.refg_insert.argtypes = [C.c_int, vp, vp, sz, vp, C.c_int]
        L.refg_insert.restype = sz
        L.refg_contains.argtypes = [C.c_int, vp, vp, sz, vp, vp]
        L.refg_delete.argtypes = [C.c_int, vp, vp, sz, vp, vp]
        L.refg_delete.restype = sz
        L.refg_clear.argtypes = [C.c_int, vp]
        L.refg_occupied.argtypes = [C.c_int, vp]
        L.refg_occupied.restype = sz
        L.refg_table.argtypes = [C.c_int, vp]
        L.refg_table.restype = vp
        L.refg_table_bytes.argtypes = [C.c_int, vp]
        L.refg_table_bytes.restype = sz
        L.refg_num_buckets.argtypes = [C.c_int, vp]
        L.refg_num_buckets.restype = sz
        _ref_gpu = L
    return _ref_gpu


class RefGpuFilter:
    """The reference's CuckooFilter<Config> (managed-memory object) on cuda:0."""

    def __init__(self, key_bytes, bits, bucket_size, policy, max_evictions, capacity, word_bytes=8,
                 alt_policy=ALT_XOR):
        key = (key_bytes, bits, bucket_size, policy, max_evictions)
        if alt_policy != ALT_XOR:
            key = key + (word_bytes, alt_policy)
        elif word_bytes != 8:
            key = key + (word_bytes,)
        self.cfg = REF_GPU_CONFIGS[key]
        self.L = ref_gpu()
        self.h = self.L.refg_create(self.cfg, capacity)
        if not self.h:
            raise RuntimeError("reference filter allocation failed")

    def close(self):
        if self.h:
            self.L.refg_destroy(self.cfg, self.h)
            self.h = None

    def insert(self, d_keys_ptr, n, stream=None, sorted_=False):
        return self.L.refg_insert(self.cfg, self.h, d_keys_ptr, n, stream, int(sorted_))

    def contains(self, d_keys_ptr, n, d_out_ptr, stream=None):
        self.L.refg_contains(self.cfg, self.h, d_keys_ptr, n, d_out_ptr, stream)

    def delete(self, d_keys_ptr, n, d_out_ptr=None, stream=None):
        return self.L.refg_delete(self.cfg, self.h, d_keys_ptr, n, d_out_ptr, stream)

    def clear(self):
        self.L.refg_clear(self.cfg, self.h)

    def occupied(self):
        return self.L.refg_occupied(self.cfg, self.h)

    def table(self):
        return self.L.refg_table(self.cfg, self.h), self.L.refg_table_bytes(self.cfg, self.h)

    def num_buckets(self):
        return self.L.refg_num_buckets(self.cfg, self.h)


def ref_candidates_policy(alt_policy, key_bytes, bits, nb, keys):
    """The reference's getCandidateBuckets for an alternate-bucket policy (bucket count nb)."""
    L = ref_host()
    k = np.ascontiguousarray(keys, dtype=np.uint64 if key_bytes == 8 else np.uint32)
    i1 = np.empty(len(k), np.uint64)
    i2 = np.empty(len(k), np.uint64)
    fp = np.empty(len(k), np.uint32)
    rc = L.ref_candidates_policy(alt_policy, key_bytes, bits, nb, _ptr(k), len(k), _ptr(i1), _ptr(i2), _ptr(fp))
    assert rc == 0
    return i1, i2, fp


def ref_alt_policy(alt_policy, bits, nb, buckets, tags):
    """The reference's alternate bucket of each (bucket, tag) and the tag as stored there."""
    L = ref_host()
    b = np.ascontiguousarray(buckets, dtype=np.uint64)
    t = np.ascontiguousarray(tags, dtype=np.uint32)
    alt = np.empty(len(b), np.uint64)
    nt = np.empty(len(b), np.uint32)
    assert L.ref_alt_policy(alt_policy, bits, nb, _ptr(b), _ptr(t), len(b), _ptr(alt), _ptr(nt)) == 0
    return alt, nt
