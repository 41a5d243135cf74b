"""B200 cuckoo filter: Python host mirror of the reference's batch API.

The names follow the reference's C++ template API (reference
``include/CuckooFilter.cuh``): ``CuckooConfig`` (:44-74) and
``CuckooFilter(config, capacity)`` (:420) with ``insertMany`` (:457),
``insertManySorted`` (:475), ``containsMany`` (:518), ``deleteMany`` (:536),
``clear`` (:675), ``loadFactor`` (:688), ``occupiedSlots`` (:699),
``capacity`` (:732), ``getNumBuckets`` (:740), ``sizeInBytes`` (:748),
``countOccupiedSlots`` (:759) and ``evictionCount`` (:714).

Every call goes through the C ABI of ``lib/libcuckoo_b200.so``
(``include/cuckoo_b200.h``) to hand-written sm_100a kernels.  There is no
other implementation: if the library is missing or no CUDA device is usable,
the calls raise.

Device memory is passed as CUDA ``torch.Tensor`` objects (torch is only the
allocator and stream provider here) or as raw device pointers (``int``) with an
explicit length.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcuckoo_b200.so")

CF_OK = 0
STATUS = {0: "CF_OK", -1: "CF_ERR_INVALID", -2: "CF_ERR_UNSUPPORTED", -3: "CF_ERR_CUDA",
          -4: "CF_ERR_NO_MEMORY", -5: "CF_ERR_DEVICE", -6: "CF_ERR_NOT_LOADED"}


class CuckooError(RuntimeError):
    """A C-ABI call returned a non-zero cf_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


# cf_option values (include/cuckoo_b200.h)
OPT_WORKSPACE_LIMIT = 1
OPT_SEGMENTED_MIN_KEYS = 2
OPT_WORKSPACE_BYTES = 3
OPT_ROUND2_SEGMENTED_MIN_KEYS = 4
OPT_REGION_MIN_KEYS = 5
OPT_STAGING = 6
OPT_REGION_BYTES = 7
OPT_REGION_COUNT = 8
OPT_LOOKUP_KPT = 9
OPT_PERSISTENT = 10
OPT_CHAIN_HISTOGRAM = 11
OPT_ROUND1_CAP = 12
OPT_PROBE_WIDTH = 13
NEVER = (1 << 64) - 1

# cf_staging values (OPT_STAGING)
STAGING_AUTO, STAGING_RANDOM, STAGING_SEGMENT, STAGING_REGION = 0, 1, 2, 3


class EvictionPolicy(enum.IntEnum):
    """Reference ``enum class EvictionPolicy`` (CuckooFilter.cuh:19-22)."""

    BFS = 0
    DFS = 1


class _Config(C.Structure):
    _fields_ = [("key_bytes", C.c_uint32), ("bits_per_tag", C.c_uint32), ("bucket_size", C.c_uint32),
                ("word_bytes", C.c_uint32), ("eviction_policy", C.c_uint32), ("max_evictions", C.c_uint32),
                ("block_size", C.c_uint32), ("alt_policy", C.c_uint32)]


class _Info(C.Structure):
    _fields_ = [("num_buckets", C.c_uint64), ("capacity", C.c_uint64), ("size_in_bytes", C.c_uint64),
                ("bucket_bytes", C.c_uint32), ("device", C.c_int32)]


class _Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("occupied", "primary", "secondary", "evicted_inserts", "evictions",
                                          "failed", "lost", "removed", "duplicates")]


_lib: Optional[C.CDLL] = None


def library() -> C.CDLL:
    """Load ``libcuckoo_b200.so`` (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python cuckoo-filter_b200/build.py`")
    L = C.CDLL(LIB_PATH)
    vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int
    P64 = C.POINTER(C.c_uint64)
    PF = C.POINTER(C.c_void_p)
    sig = {
        "cf_abi_version": ([], i32),
        "cf_launch_count": ([], u64),
        "cf_get_chain_histogram": ([vp, vp], i32),
        "cf_last_error": ([], C.c_char_p),
        "cf_status_string": ([i32], C.c_char_p),
        "cf_config_supported": ([C.POINTER(_Config)], i32),
        "cf_num_buckets_for": ([u64, u32], u64),
        "cf_num_buckets_for_policy": ([u64, u32, u32], u64),
        "cf_create": ([C.POINTER(_Config), u64, PF], i32),
        "cf_destroy": ([vp], i32),
        "cf_get_info": ([vp, C.POINTER(_Info)], i32),
        "cf_insert": ([vp, vp, u64, vp, vp, P64], i32),
        "cf_insert_sorted": ([vp, vp, u64, vp, vp, P64], i32),
        "cf_contains": ([vp, vp, u64, vp, vp], i32),
        "cf_delete": ([vp, vp, u64, vp, vp, P64], i32),
        "cf_insert_async": ([vp, vp, u64, vp, vp], i32),
        "cf_contains_async": ([vp, vp, u64, vp, vp], i32),
        "cf_delete_async": ([vp, vp, u64, vp, vp], i32),
        "cf_clear": ([vp, vp], i32),
        "cf_occupied": ([vp, P64], i32),
        "cf_count_occupied_slots": ([vp, P64], i32),
        "cf_get_stats": ([vp, C.POINTER(_Stats)], i32),
        "cf_reset_stats": ([vp], i32),
        "cf_table": ([vp, PF, P64], i32),
        "cf_load_table": ([vp, vp, u64, vp], i32),
        "cf_store_table": ([vp, vp, u64, vp], i32),
        "cf_probe_count": ([vp, vp, u64, P64, vp], i32),
        "cf_hash_candidates": ([C.POINTER(_Config), u64, vp, u64, vp, vp, vp], i32),
        "cf_hash64": ([u32, vp, u64, vp], i32),
        "cf_set_create": ([C.POINTER(_Config), u32, vp, PF], i32),
        "cf_set_destroy": ([vp], i32),
        "cf_set_size": ([vp, C.POINTER(C.c_uint32), P64], i32),
        "cf_set_get_info": ([vp, u32, C.POINTER(_Info)], i32),
        "cf_set_table": ([vp, u32, PF, P64], i32),
        "cf_set_insert_async": ([vp, vp, u64, vp, vp, u32, vp, vp], i32),
        "cf_set_contains_async": ([vp, vp, u64, vp, vp, u32, vp, vp], i32),
        "cf_set_delete_async": ([vp, vp, u64, vp, vp, u32, vp, vp], i32),
        "cf_set_sync": ([vp, vp], i32),
        "cf_set_clear": ([vp, vp], i32),
        "cf_set_occupied": ([vp, vp], i32),
        "cf_set_get_stats": ([vp, u32, C.POINTER(_Stats)], i32),
        "cf_set_set_launch": ([vp, i32, u32, u32, u32], i32),
        "cf_set_get_launch": ([vp, i32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)], i32),
        "cf_set_autotune": ([vp, i32, vp, u64, vp, vp, u32, vp, vp, C.POINTER(C.c_float)], i32),
        "cf_insert_sorted_noalloc": ([vp, vp, u64, vp, vp, P64], i32),
        "cf_noalloc_scratch_bytes": ([], u64),
        "cf_alt_buckets": ([C.POINTER(_Config), u64, vp, vp, u64, vp], i32),
        "cf_set_option": ([vp, i32, u64], i32),
        "cf_get_option": ([vp, i32, P64], i32),
        "cf_shard_workspace_bytes": ([u64, u32], u64),
        "cf_shard_partition": ([vp, u64, u32, u32, u32, vp, vp, vp, vp, u64, vp], i32),
        "cf_shard_unpartition": ([vp, vp, u64, u32, vp, u64, vp, vp], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def launch_count() -> int:
    """Kernels the library has launched since it was loaded."""
    return int(library().cf_launch_count())


def _check(status: int) -> None:
    if status != CF_OK:
        raise CuckooError(status, library().cf_last_error().decode(errors="replace"))


_KEY_BYTES = {"uint64": 8, "uint64_t": 8, "int64": 8, "uint32": 4, "uint32_t": 4, "int32": 4}

ALT_XOR, ALT_ADDSUB, ALT_OFFSET = 0, 1, 2
_ALT_POLICIES = {"XorAltBucketPolicy": ALT_XOR, "xor": ALT_XOR, "AddSubAltBucketPolicy": ALT_ADDSUB,
                 "addsub": ALT_ADDSUB, "OffsetAltBucketPolicy": ALT_OFFSET, "offset": ALT_OFFSET}


@dataclass(frozen=True)
class CuckooConfig:
    """Runtime form of ``CuckooConfig<T, bitsPerTag, maxEvictions, blockSize,
    bucketSize, AltBucketPolicy, evictionPolicy, WordType>`` (CuckooFilter.cuh:44-74).

    Defaults are the reference's template defaults (maxEvictions 500, blockSize
    256, bucketSize 16, XorAltBucketPolicy, DFS, uint64_t words).
    """

    T: str
    bitsPerTag: int
    maxEvictions: int = 500
    blockSize: int = 256
    bucketSize: int = 16
    AltBucketPolicy: str = "XorAltBucketPolicy"
    evictionPolicy: EvictionPolicy = EvictionPolicy.DFS
    WordType: str = "uint64_t"

    @property
    def key_bytes(self) -> int:
        return _KEY_BYTES[str(self.T).replace("torch.", "").replace("np.", "")]

    @property
    def TagType(self) -> str:
        return "uint8_t" if self.bitsPerTag <= 8 else "uint16_t" if self.bitsPerTag <= 16 else "uint32_t"

    @property
    def alt_policy(self) -> int:
        """cf_alt_policy of AltBucketPolicy (XorAltBucketPolicy, AddSubAltBucketPolicy or OffsetAltBucketPolicy)."""
        try:
            return _ALT_POLICIES[self.AltBucketPolicy]
        except KeyError:
            raise CuckooError(-1, f"unknown alternate-bucket policy {self.AltBucketPolicy}") from None

    def to_c(self) -> _Config:
        word = {"uint64_t": 8, "uint64": 8, "uint32_t": 4, "uint32": 4}[self.WordType]
        return _Config(self.key_bytes, self.bitsPerTag, self.bucketSize, word, int(self.evictionPolicy),
                       self.maxEvictions, self.blockSize, self.alt_policy)


def _torch():
    import torch

    return torch


def _dev_ptr(x, n: Optional[int], elem_bytes: int, what: str):
    """(pointer, n) of a CUDA tensor or a raw device pointer."""
    if isinstance(x, int):
        if n is None:
            raise ValueError(f"{what}: a raw pointer needs an explicit length")
        return x, n
    torch = _torch()
    if not isinstance(x, torch.Tensor):
        raise TypeError(f"{what}: expected a CUDA tensor or a device pointer, got {type(x).__name__}")
    if not x.is_cuda:
        raise ValueError(f"{what}: tensor must be on a CUDA device")
    if not x.is_contiguous():
        raise ValueError(f"{what}: tensor must be contiguous")
    if x.element_size() != elem_bytes:
        raise ValueError(f"{what}: element size {x.element_size()} != {elem_bytes}")
    return x.data_ptr(), (x.numel() if n is None else n)


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream or None
    if isinstance(stream, int):
        return stream or None
    return stream.cuda_stream or None


class CuckooFilter:
    """The filter; owns its device table.  Mirrors ``CuckooFilter<Config>``."""

    def __init__(self, config: CuckooConfig, capacity: int):
        self.config = config
        L = library()
        h = C.c_void_p()
        c = config.to_c()
        _check(L.cf_create(C.byref(c), int(capacity), C.byref(h)))
        self._h = h
        info = _Info()
        _check(L.cf_get_info(self._h, C.byref(info)))
        self.numBuckets = int(info.num_buckets)
        self._capacity = int(info.capacity)
        self._bytes = int(info.size_in_bytes)
        self.bucketBytes = int(info.bucket_bytes)
        self.device = int(info.device)

    # -------------------------------------------------------------- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            library().cf_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return int(self._h.value or 0)

    # ------------------------------------------------------------ batch ops
    def insertMany(self, d_keys, n: Optional[int] = None, stream=None, d_output=None) -> int:
        """Insert keys; returns occupiedSlots() after the batch (CuckooFilter.cuh:457)."""
        ptr, n = _dev_ptr(d_keys, n, self.config.key_bytes, "d_keys")
        out = 0 if d_output is None else _dev_ptr(d_output, n, 1, "d_output")[0]
        occ = C.c_uint64()
        _check(library().cf_insert(self._h, ptr, n, out or None, _stream_handle(stream), C.byref(occ)))
        return int(occ.value)

    def insertManySorted(self, d_keys, n: Optional[int] = None, stream=None, d_output=None) -> int:
        """Insert keys partitioned by primary bucket (CuckooFilter.cuh:475)."""
        ptr, n = _dev_ptr(d_keys, n, self.config.key_bytes, "d_keys")
        out = 0 if d_output is None else _dev_ptr(d_output, n, 1, "d_output")[0]
        occ = C.c_uint64()
        _check(library().cf_insert_sorted(self._h, ptr, n, out or None, _stream_handle(stream), C.byref(occ)))
        return int(occ.value)

    def containsMany(self, d_keys, d_output=None, n: Optional[int] = None, stream=None):
        """Membership of each key (CuckooFilter.cuh:518).  Returns the output tensor."""
        ptr, n = _dev_ptr(d_keys, n, self.config.key_bytes, "d_keys")
        if d_output is None:
            torch = _torch()
            d_output = torch.empty(n, dtype=torch.bool, device=f"cuda:{self.device}")
        optr, _ = _dev_ptr(d_output, n, 1, "d_output")
        _check(library().cf_contains(self._h, ptr, n, optr, _stream_handle(stream)))
        return d_output

    def deleteMany(self, d_keys, d_output=None, n: Optional[int] = None, stream=None) -> int:
        """Remove one copy per key; returns occupiedSlots() (CuckooFilter.cuh:536)."""
        ptr, n = _dev_ptr(d_keys, n, self.config.key_bytes, "d_keys")
        out = 0 if d_output is None else _dev_ptr(d_output, n, 1, "d_output")[0]
        occ = C.c_uint64()
        _check(library().cf_delete(self._h, ptr, n, out or None, _stream_handle(stream), C.byref(occ)))
        return int(occ.value)

    # asynchronous forms (no synchronisation, no return value)
    def insertManyAsync(self, d_keys, n=None, stream=None, d_output=None) -> None:
        ptr, n = _dev_ptr(d_keys, n, self.config.key_bytes, "d_keys")
        out = 0 if d_output is None else _dev_ptr(d_output, n, 1, "d_output")[0]
        _check(library().cf_insert_async(self._h, ptr, n, out or None, _stream_handle(stream)))

    def containsManyAsync(self, d_keys, d_output, n=None, stream=None) -> None:
        ptr, n = _dev_ptr(d_keys, n, self.config.key_bytes, "d_keys")
        optr, _ = _dev_ptr(d_output, n, 1, "d_output")
        _check(library().cf_contains_async(self._h, ptr, n, optr, _stream_handle(stream)))

    def deleteManyAsync(self, d_keys, d_output=None, n=None, stream=None) -> None:
        ptr, n = _dev_ptr(d_keys, n, self.config.key_bytes, "d_keys")
        out = 0 if d_output is None else _dev_ptr(d_output, n, 1, "d_output")[0]
        _check(library().cf_delete_async(self._h, ptr, n, out or None, _stream_handle(stream)))

    # ---------------------------------------------------------- bookkeeping
    def clear(self, stream=None) -> None:
        _check(library().cf_clear(self._h, _stream_handle(stream)))

    def occupiedSlots(self) -> int:
        v = C.c_uint64()
        _check(library().cf_occupied(self._h, C.byref(v)))
        return int(v.value)

    def loadFactor(self) -> float:
        import numpy as np

        return float(np.float32(self.occupiedSlots()) / np.float32(self._capacity))

    def capacity(self) -> int:
        return self._capacity

    def getNumBuckets(self) -> int:
        return self.numBuckets

    def sizeInBytes(self) -> int:
        return self._bytes

    def countOccupiedSlots(self) -> int:
        v = C.c_uint64()
        _check(library().cf_count_occupied_slots(self._h, C.byref(v)))
        return int(v.value)

    def setOption(self, option: int, value: int) -> None:
        """cf_set_option: OPT_WORKSPACE_LIMIT (bytes) or OPT_SEGMENTED_MIN_KEYS (0 = automatic)."""
        _check(library().cf_set_option(self._h, option, value))

    def getOption(self, option: int) -> int:
        v = C.c_uint64()
        _check(library().cf_get_option(self._h, option, C.byref(v)))
        return int(v.value)

    def stats(self) -> dict:
        s = _Stats()
        _check(library().cf_get_stats(self._h, C.byref(s)))
        return {name: int(getattr(s, name)) for name, _ in _Stats._fields_}

    def chainHistogram(self):
        """Eviction-chain-length histogram (CF_CHAIN_BINS bins; see cuckoo_b200.h)."""
        import numpy as np

        out = np.zeros(10, np.uint64)
        _check(library().cf_get_chain_histogram(self._h, out.ctypes.data))
        return out

    def evictionCount(self) -> int:
        return self.stats()["evictions"]

    def resetEvictionCount(self) -> None:
        _check(library().cf_reset_stats(self._h))

    def table(self):
        """(device pointer, bytes) of the table image."""
        p = C.c_void_p()
        b = C.c_uint64()
        _check(library().cf_table(self._h, C.byref(p), C.byref(b)))
        return int(p.value or 0), int(b.value)

    def table_image(self, device: Optional[str] = None):
        """Copy of the table image as a uint8 tensor (on the filter's GPU by default)."""
        torch = _torch()
        out = torch.empty(self._bytes, dtype=torch.uint8, device=device or f"cuda:{self.device}")
        _check(library().cf_store_table(self._h, out.data_ptr(), self._bytes, _stream_handle(None)))
        return out

    def load_table(self, image, nbytes: Optional[int] = None) -> None:
        """Replace the table with an image (a CUDA/CPU tensor, or a device pointer
        with ``nbytes``) and recount the occupancy."""
        if isinstance(image, int):
            ptr, n = image, nbytes
        else:
            ptr, n = image.data_ptr(), image.numel() * image.element_size()
        _check(library().cf_load_table(self._h, ptr, n, _stream_handle(None)))

    def store_table(self, dst: int, nbytes: int) -> None:
        """Copy the table image to a raw (device or host) pointer."""
        _check(library().cf_store_table(self._h, dst, nbytes, _stream_handle(None)))

    def probe_count(self, d_keys, n: Optional[int] = None, stream=None) -> int:
        ptr, n = _dev_ptr(d_keys, n, self.config.key_bytes, "d_keys")
        v = C.c_uint64()
        _check(library().cf_probe_count(self._h, ptr, n, C.byref(v), _stream_handle(stream)))
        return int(v.value)

    # ------------------------------------------------------ static helpers
    @staticmethod
    def calculateNumBuckets(capacity: int, bucketSize: int = 16, AltBucketPolicy: str = "XorAltBucketPolicy") -> int:
        """The policy's calculateNumBuckets (bucket_policies.cuh:80-83, :166-176, :346-349)."""
        return int(library().cf_num_buckets_for_policy(capacity, bucketSize, _ALT_POLICIES[AltBucketPolicy]))

    @staticmethod
    def getCandidateBuckets(config: CuckooConfig, keys, numBuckets: int):
        """(i1, i2, fp) arrays for host keys (the configured policy's getCandidateBuckets;
        fp as stored in the primary bucket)."""
        import numpy as np

        k = np.ascontiguousarray(keys, dtype=np.uint64 if config.key_bytes == 8 else np.uint32)
        i1 = np.empty(len(k), np.uint64)
        i2 = np.empty(len(k), np.uint64)
        fp = np.empty(len(k), np.uint32)
        c = config.to_c()
        _check(library().cf_hash_candidates(C.byref(c), numBuckets, k.ctypes.data, len(k), i1.ctypes.data,
                                            i2.ctypes.data, fp.ctypes.data))
        return i1, i2, fp


SET_INSERT, SET_CONTAINS, SET_DELETE = 0, 1, 2


class CuckooFilterSet:
    """Many independent filters of one configuration, batched (cf_set_* ABI).

    A batched call takes the concatenated keys of all items plus a device work
    list: ``offsets`` (int64, n_items + 1 entries, offsets[-1] == len(keys))
    and ``filters`` (int32, n_items): item j is keys[offsets[j]:offsets[j+1]]
    for filter filters[j].  Every item runs in one kernel launch.  The
    ``*_async`` methods only enqueue (capturable in a CUDA graph); ``sync()``
    waits and raises on device-side errors.
    """

    def __init__(self, config: CuckooConfig, capacities):
        import numpy as np

        self.config = config
        caps = np.ascontiguousarray(np.asarray(capacities, dtype=np.uint64))
        h = C.c_void_p()
        c = config.to_c()
        _check(library().cf_set_create(C.byref(c), len(caps), caps.ctypes.data, C.byref(h)))
        self._h = h
        self.n = len(caps)
        info = _Info()
        self.num_buckets = []
        self.capacities = []
        for i in range(self.n):
            _check(library().cf_set_get_info(self._h, i, C.byref(info)))
            self.num_buckets.append(int(info.num_buckets))
            self.capacities.append(int(info.capacity))
        self.device = int(info.device)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            library().cf_set_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return int(self._h.value or 0)

    def _args(self, keys, offsets, filters, out):
        kp, n = _dev_ptr(keys, None, 8, "keys")
        op, no = _dev_ptr(offsets, None, 8, "offsets")
        fp, nf = _dev_ptr(filters, None, 4, "filters")
        if no != nf + 1:
            raise ValueError("offsets must have len(filters) + 1 entries")
        optr = 0 if out is None else _dev_ptr(out, n, 1, "out")[0]
        return kp, n, op, fp, nf, optr or None

    def insert_async(self, keys, offsets, filters, out=None, stream=None) -> None:
        kp, n, op, fp, nf, optr = self._args(keys, offsets, filters, out)
        _check(library().cf_set_insert_async(self._h, kp, n, op, fp, nf, optr, _stream_handle(stream)))

    def contains_async(self, keys, offsets, filters, out, stream=None) -> None:
        kp, n, op, fp, nf, optr = self._args(keys, offsets, filters, out)
        _check(library().cf_set_contains_async(self._h, kp, n, op, fp, nf, optr, _stream_handle(stream)))

    def delete_async(self, keys, offsets, filters, out=None, stream=None) -> None:
        kp, n, op, fp, nf, optr = self._args(keys, offsets, filters, out)
        _check(library().cf_set_delete_async(self._h, kp, n, op, fp, nf, optr, _stream_handle(stream)))

    def sync(self, stream=None) -> None:
        _check(library().cf_set_sync(self._h, _stream_handle(stream)))

    def clear(self, stream=None) -> None:
        _check(library().cf_set_clear(self._h, _stream_handle(stream)))

    def occupied(self):
        import numpy as np

        out = np.zeros(self.n, np.uint64)
        _check(library().cf_set_occupied(self._h, out.ctypes.data))
        return out

    def stats(self, i: int) -> dict:
        st = _Stats()
        _check(library().cf_set_get_stats(self._h, i, C.byref(st)))
        return {name: int(getattr(st, name)) for name, _ in _Stats._fields_}

    def table(self, i: int):
        p = C.c_void_p()
        b = C.c_uint64()
        _check(library().cf_set_table(self._h, i, C.byref(p), C.byref(b)))
        return int(p.value or 0), int(b.value)

    def table_view(self, i: int):
        """Filter i's table image as a uint8 CUDA tensor viewing the set's pool
        (no copy; valid while the set lives)."""
        ptr, nbytes = self.table(i)
        return _device_view(ptr, nbytes, self.device)

    def table_image(self, i: int):
        """Copy of filter i's table image as a uint8 CPU tensor."""
        return self.table_view(i).cpu()

    def load_table(self, i: int, image) -> None:
        """Replace filter i's table with an image (CPU or CUDA uint8 tensor).
        Counters are not recomputed."""
        view = self.table_view(i)
        if image.numel() != view.numel():
            raise ValueError(f"image is {image.numel()} bytes, table is {view.numel()}")
        view.copy_(image)
        _torch().cuda.synchronize(self.device)

    def set_launch(self, op: int, block: int, kpt: int, width: int = 1) -> None:
        _check(library().cf_set_set_launch(self._h, op, block, kpt, width))

    def get_launch(self, op: int):
        b, k, w = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(library().cf_set_get_launch(self._h, op, C.byref(b), C.byref(k), C.byref(w)))
        return int(b.value), int(k.value), int(w.value)

    def autotune(self, op: int, keys, offsets, filters, out=None, stream=None) -> float:
        kp, n, opp, fp, nf, optr = self._args(keys, offsets, filters, out)
        best = C.c_float()
        _check(library().cf_set_autotune(self._h, op, kp, n, opp, fp, nf, optr, _stream_handle(stream),
                                         C.byref(best)))
        return float(best.value)


class _DeviceBuffer:
    """Raw device memory exposed through __cuda_array_interface__."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 2}


def _device_view(ptr: int, nbytes: int, device: int):
    torch = _torch()
    return torch.as_tensor(_DeviceBuffer(ptr, nbytes), device=f"cuda:{device}")


__all__ = ["CuckooConfig", "CuckooFilter", "CuckooFilterSet", "EvictionPolicy", "CuckooError", "library", "LIB_PATH"]
