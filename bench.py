#!/usr/bin/env python3
"""Benchmark of the cuckoo filter batch path on B200.

Metric: Gkeys/s of insert + lookup (+ delete) at 95 % load, with each kernel's
fraction of the HBM sector roofline.  One step = clear the filter, insertMany
the fill keys (to 0.95 load), containsMany a 50 %-positive batch, deleteMany a
batch of stored keys.

Default workload ("large"): 2^31 slots, 16-bit tags, 16-slot buckets (4 GiB
table), BFS eviction, maxEvictions 500, uint64 keys; fill = floor(0.95 * 2^31)
keys from splitmix64(seed 3); 2^28 lookups = 2^27 stored keys sampled without
replacement + 2^27 splitmix64(seed 4) keys that are not stored; 2^26 deletes
(the first 2^26 sampled stored keys).  Every input is larger than the 126 MB L2.

Legs of one run:
  value       device-resident inputs; CUDA events around each step on the
              launching stream; async C-ABI calls (one kernel per op).
  e2e         the synchronous C-ABI calls (insertMany/containsMany/deleteMany)
              with inputs copied from pinned host memory and results copied
              back inside the timed region.
  cpu_baseline the oracle's multithreaded CPU port on a bounded sample.

`--impl reference` times the reference's algorithm on the host cores (the CPU
port, all threads) on a bounded sample of the same workload and, where the
reference's own CUDA kernels were built (oracle/_ref), those kernels on the
full workload on this GPU.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import random
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Gkeys/s insert & lookup at 95% load, % of HBM sector roofline; p99 req latency"

G = 0x9E3779B97F4A7C15
M1 = 0xBF58476D1CE4E5B9
M2 = 0x94D049BB133111EB
U64 = 1 << 64

WORKLOADS = {
    "large": dict(
        desc="large out-of-L2 filter: 2^31 slots, 16-bit tags, 16-slot buckets (4 GiB), BFS, maxEvictions 500, "
             "uint64 keys; fill 0.95 (splitmix64 seed 3); 2^28 lookups 50% positive; 2^26 deletes",
        capacity=1 << 31, bits=16, bs=16, policy="BFS", max_ev=500, fill=0.95,
        n_pos=1 << 27, n_neg=1 << 27, n_del=1 << 26, seed_fill=3, seed_neg=4, seed_sample=5),
    "medium": dict(
        desc="medium out-of-L2 filter for profiling: 2^28 slots, 16-bit tags, 16-slot buckets (512 MiB), BFS; "
             "fill 0.95 (splitmix64 seed 3); 2^25 lookups 50% positive; 2^23 deletes",
        capacity=1 << 28, bits=16, bs=16, policy="BFS", max_ev=500, fill=0.95,
        n_pos=1 << 24, n_neg=1 << 24, n_del=1 << 23, seed_fill=3, seed_neg=4, seed_sample=5),
    "small": dict(
        desc="small filter (L2-resident): 2^20 slots, 16-bit tags, 16-slot buckets, BFS; 996147 keys "
             "(splitmix64 seed 1); lookups of all of them + 996147 negatives (seed 2); delete half",
        capacity=1 << 20, bits=16, bs=16, policy="BFS", max_ev=500, fill=0.95,
        n_pos=996147, n_neg=996147, n_del=996147 // 2, seed_fill=1, seed_neg=2, seed_sample=0),
}


def s64(x: int) -> int:
    x %= U64
    return x - U64 if x >= (1 << 63) else x


# ------------------------------------------------------------------ inputs


def splitmix64_torch(seed: int, first: int, n: int, out, chunk: int = 1 << 27):
    """splitmix64 outputs first..first+n-1 of `seed` into an int64 tensor (any device).

    Output i is mix(seed + (i+1) * 0x9E3779B97F4A7C15) with the published
    splitmix64 finaliser; int64 arithmetic wraps modulo 2^64.
    """
    import torch

    def lsr(z, s):
        return (z >> s) & ((1 << (64 - s)) - 1)

    for off in range(0, n, chunk):
        m = min(chunk, n - off)
        i = torch.arange(first + off + 1, first + off + 1 + m, device=out.device, dtype=torch.int64)
        z = i * s64(G) + s64(seed)
        z = (z ^ lsr(z, 30)) * s64(M1)
        z = (z ^ lsr(z, 27)) * s64(M2)
        out[off:off + m] = z ^ lsr(z, 31)
    return out


# ------------------------------------------- parity check: hashing and digests
#
# An independent restatement, in torch int64 arithmetic, of the reference's
# key hashing (xxHash64 with seed 0 over the value's little-endian bytes,
# reference include/hashutil.cuh:71-161) and of XorAltBucketPolicy
# (bucket_policies.cuh:46-74).  It shares no code with the library's kernels,
# so it can check a table the kernels built; tests pin it to the golden vectors
# made from the reference's own headers.  int64 products wrap modulo 2^64.

XXH_P1, XXH_P2, XXH_P3 = 0x9E3779B185EBCA87, 0xC2B2AE3D27D4EB4F, 0x165667B19E3779F9
XXH_P4, XXH_P5 = 0x85EBCA77C2B2AE63, 0x27D4EB2F165667C5


def _lsr(z, s: int):
    return (z >> s) & ((1 << (64 - s)) - 1)


def _rotl(z, r: int):
    return (z << r) | _lsr(z, 64 - r)


def _xxh_avalanche(h):
    h = (h ^ _lsr(h, 33)) * s64(XXH_P2)
    h = (h ^ _lsr(h, 29)) * s64(XXH_P3)
    return h ^ _lsr(h, 32)


def xxh64_torch(v, nbytes: int):
    """XXH64 (seed 0) of each value of the int64 tensor `v`, read as `nbytes`
    (1, 2, 4 or 8) little-endian bytes."""
    h = v * 0 + s64(XXH_P5 + nbytes)
    if nbytes == 8:
        k1 = _rotl(v * s64(XXH_P2), 31) * s64(XXH_P1)
        h = _rotl(h ^ k1, 27) * s64(XXH_P1) + s64(XXH_P4)
    elif nbytes == 4:
        h = _rotl(h ^ ((v & 0xFFFFFFFF) * s64(XXH_P1)), 23) * s64(XXH_P2) + s64(XXH_P3)
    else:
        for i in range(nbytes):
            h = _rotl(h ^ (((v >> (8 * i)) & 0xFF) * s64(XXH_P5)), 11) * s64(XXH_P1)
    return _xxh_avalanche(h)


def tag_hash_table(bits: int, device):
    """xxHash64 of every tag value of a bits-bit TagType (8 or 16 bits) as a lookup table."""
    import torch

    return xxh64_torch(torch.arange(1 << bits, dtype=torch.int64, device=device), bits // 8)


def candidates_torch(keys, key_bytes: int, bits: int, num_buckets: int, tag_lut=None):
    """(i1, i2, fp) of XorAltBucketPolicy::getCandidateBuckets: fp from the
    upper 32 hash bits masked to `bits` (0 becomes 1), i1 from the lower 32 bits
    masked to the bucket count, i2 = i1 ^ (xxHash64(fp as TagType) & (nB - 1))."""
    h = xxh64_torch(keys if key_bytes == 8 else keys & 0xFFFFFFFF, key_bytes)
    fp = _lsr(h, 32) & ((1 << bits) - 1)
    fp = fp + (fp == 0).to(fp.dtype)
    mask = num_buckets - 1
    i1 = h & 0xFFFFFFFF & mask
    th = tag_lut[fp] if tag_lut is not None else xxh64_torch(fp, bits // 8)
    return i1, i1 ^ (th & mask), fp


_DIGEST_SEEDS = (0x2545F4914F6CDD1D, 0x7FB5D329728EA185)


def _digest_add(acc: list, sig, valid) -> None:
    """acc += (count, sum of two 32-bit mixes) over sig[valid], exactly (Python ints)."""
    import torch

    sig = sig[valid]
    acc[0] += int(sig.numel())
    for j, seed in enumerate(_DIGEST_SEEDS):
        z = sig + s64(seed)
        z = (z ^ _lsr(z, 30)) * s64(M1)
        z = (z ^ _lsr(z, 27)) * s64(M2)
        acc[1 + j] += int(_lsr(z ^ _lsr(z, 31), 32).sum(dtype=torch.int64).item())


def key_digest(keys, bits: int, num_buckets: int, valid=None, chunk: int = 1 << 26) -> tuple:
    """Multiset digest of the (bucket pair, tag) entries that storing `keys`
    (int64 tensor of 8-byte keys; rows with valid == False skipped) must leave in
    the table: per key, (min(i1, i2) << bits) | fp, mixed and summed."""
    import torch

    lut = tag_hash_table(bits, keys.device) if bits <= 16 else None
    acc = [0, 0, 0]
    for a in range(0, keys.numel(), chunk):
        k = keys[a:a + chunk]
        i1, i2, fp = candidates_torch(k, 8, bits, num_buckets, lut)
        v = valid[a:a + chunk] if valid is not None else torch.ones_like(fp, dtype=torch.bool)
        _digest_add(acc, (torch.minimum(i1, i2) << bits) | fp, v)
    return tuple(acc)


def table_digest(table_u8, bits: int, bucket_size: int, num_buckets: int, chunk_slots: int = 1 << 26) -> tuple:
    """Multiset digest of the table image (uint8 tensor, the reference's layout):
    for every occupied slot of bucket b holding tag t, (min(b, alt(b, t)) << bits) | t."""
    import torch

    view = {8: torch.uint8, 16: torch.int16, 32: torch.int32}[bits]
    slots = table_u8.view(view)
    lut = tag_hash_table(bits, slots.device) if bits <= 16 else None
    mask = num_buckets - 1
    acc = [0, 0, 0]
    per = chunk_slots // bucket_size * bucket_size
    for a in range(0, slots.numel(), per):
        t = slots[a:a + per].to(torch.int64) & ((1 << bits) - 1)
        b = (torch.arange(t.numel(), device=t.device, dtype=torch.int64) + a) // bucket_size
        th = lut[t] if lut is not None else xxh64_torch(t, 4)
        _digest_add(acc, (torch.minimum(b, b ^ (th & mask)) << bits) | t, t != 0)
    return tuple(acc)


def digest_sub(a: tuple, b: tuple) -> tuple:
    """Digest of multiset a minus multiset b (b contained in a)."""
    return tuple(x - y for x, y in zip(a, b))


def negative_collisions(seed_pos: int, n_pos: int, seed_neg: int, n_neg: int) -> list[int]:
    """Indices j of splitmix64(seed_neg) outputs equal to some splitmix64(seed_pos)
    output with index < n_pos.  splitmix64 is a bijection of its state, so
    outputs are equal iff states are: j collides with i = j + c (mod 2^64),
    c = (seed_neg - seed_pos) / gamma (mod 2^64)."""
    c = ((seed_neg - seed_pos) * pow(G, -1, U64)) % U64
    out: list[int] = []
    # i = (j + c) mod 2^64 < n_pos  <=>  j in [(-c) mod 2^64, (-c) mod 2^64 + n_pos), modulo 2^64
    lo = (-c) % U64
    for j0 in (lo, lo - U64):
        a, b = max(0, j0), min(n_neg, j0 + n_pos)
        if a < b:
            out.extend(range(a, b))
    return out


def collides(seed_pos: int, n_pos: int, seed_neg: int, j: int) -> bool:
    c = ((seed_neg - seed_pos) * pow(G, -1, U64)) % U64
    return (j + c) % U64 < n_pos


def make_inputs(w: dict, device, rank: int = 0, with_mask: bool = False):
    """Device tensors: fill keys, query keys (positives and negatives shuffled),
    delete keys, the number of negatives replaced; with `with_mask` also a bool
    tensor marking the positives of the query batch."""
    import torch

    seed_fill = w["seed_fill"] + 1000 * rank
    seed_neg = w["seed_neg"] + 1000 * rank
    n_fill = int(w["fill"] * w["capacity"])
    fill = torch.empty(n_fill, dtype=torch.int64, device=device)
    splitmix64_torch(seed_fill, 0, n_fill, fill)
    n_pos, n_neg = w["n_pos"], w["n_neg"]
    if n_pos >= n_fill:
        pos = fill[:n_pos]
    else:
        # sample without replacement: j -> (a*j + b) mod n_fill, gcd(a, n_fill) = 1
        r = random.Random(w["seed_sample"] + rank)
        while True:
            a = r.randrange(1, n_fill)
            if math.gcd(a, n_fill) == 1:
                break
        b = r.randrange(0, n_fill)
        j = torch.arange(n_pos, device=device, dtype=torch.int64)
        pos = fill[(j * a + b) % n_fill]
    neg = torch.empty(n_neg, dtype=torch.int64, device=device)
    splitmix64_torch(seed_neg, 0, n_neg, neg)
    bad = negative_collisions(seed_fill, n_fill, seed_neg, n_neg)
    extra = n_neg
    for j in bad:  # replace colliding negatives by later outputs of the same stream
        while collides(seed_fill, n_fill, seed_neg, extra):
            extra += 1
        cand = torch.empty(1, dtype=torch.int64, device=device)
        splitmix64_torch(seed_neg, extra, 1, cand)
        extra += 1
        neg[j] = cand[0]
    g = torch.Generator(device=device)
    g.manual_seed(w["seed_sample"] + 17 + rank)
    query = torch.cat([pos, neg])
    perm = torch.randperm(query.numel(), generator=g, device=device)
    query = query[perm]
    dele = pos[: w["n_del"]].clone()
    if with_mask:
        return fill, query, dele, len(bad), perm < n_pos
    return fill, query, dele, len(bad)


# ------------------------------------------------------------------ helpers


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.05)  # the sample in progress, not the idle time after the region
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in getattr(self, "lines", []):
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


_REGISTERED = []


def pinned_empty(n: int, dtype):
    """Host tensor in page-locked memory.  Registers an ordinary allocation
    (cudaHostRegister) instead of using torch's pinned allocator, which rounds
    sizes up to a power of two."""
    import torch

    t = torch.empty(n, dtype=dtype)
    nbytes = t.numel() * t.element_size()
    if nbytes and torch._C._cudart.cudaHostRegister(t.data_ptr(), nbytes, 0) == 0:
        _REGISTERED.append(t)
        return t
    return torch.empty(n, dtype=dtype, pin_memory=True)


def release_pinned() -> None:
    import torch

    while _REGISTERED:
        t = _REGISTERED.pop()
        torch._C._cudart.cudaHostUnregister(t.data_ptr())


def measured_peak() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _reduce(world, x: float, op: str) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(world, x: float) -> float:
    return _reduce(world, x, "max")


def sum_over_ranks(world, x: float) -> float:
    return _reduce(world, x, "sum")


def aggregate(world, keys_per_step: int, steps: int, total_ms: float) -> tuple[float, float]:
    """Whole-job throughput: keys processed by all ranks (each rank owns an
    independent filter shard) over the slowest rank's device time.  Returns
    (Gkeys/s, max total ms)."""
    total_ms_max = max_over_ranks(world, total_ms)
    all_keys = sum_over_ranks(world, keys_per_step * steps)
    return all_keys / (total_ms_max / 1e3) / 1e9, total_ms_max


# ------------------------------------------------------------ CPU baselines


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


class CpuFullTable:
    """The reference's algorithm on the host cores (the oracle's port of
    CuckooFilter.cuh:805-1116 with atomic compare-and-swap on 64-bit words,
    oracle/cf_oracle.c) on the workload's full-size table.

    fill(): the whole fill once, in 20 load strata; in each stratum the first
    1/64 of its keys is inserted by one thread and the rest by all threads, so
    both rates are averaged over the same 0 -> 0.95 load range.
    step(k): on the full table at 0.95 load, slice k of the lookup batch and of
    the delete batch by all threads and a 1/16 sub-slice by one thread (deleted
    keys are re-inserted, untimed, so every step sees the same table).
    Rates combine as the workload's own mix: (fill + lookups + deletes) keys
    over fill / r_insert + lookups / r_lookup + deletes / r_delete."""

    STRATA, ONE_IN = 20, 64

    def __init__(self, w: dict, fill, query, dele, threads: int, q_slice: int = 1 << 22, d_slice: int = 1 << 20):
        import oracle

        self.oracle = oracle
        self.L = oracle.lib()
        pol = oracle.POLICY_BFS if w["policy"] == "BFS" else oracle.POLICY_DFS
        self.o = oracle.OracleFilter(key_bytes=8, bits=w["bits"], bucket_size=w["bs"], policy=pol,
                                     max_evictions=w["max_ev"], capacity=w["capacity"])
        self.fill_keys, self.query, self.dele = fill, query, dele
        self.threads = threads
        self.q_slice, self.d_slice = min(q_slice, len(query)), min(d_slice, len(dele))
        self.n = (len(fill), len(query), len(dele))
        self.rates = {}

    def _run(self, fn, keys, a: int, m: int, threads: int) -> float:
        import ctypes as C

        t0 = time.perf_counter()
        fn(C.byref(self.o.p), self.o.table.ctypes.data, keys.ctypes.data + 8 * a, m, None, threads)
        return time.perf_counter() - t0

    def fill(self) -> None:
        n = len(self.fill_keys)
        t1 = tn = 0.0
        n1 = nn = 0
        for k in range(self.STRATA):
            a, b = k * n // self.STRATA, (k + 1) * n // self.STRATA
            s = max(1, (b - a) // self.ONE_IN)
            t1 += self._run(self.L.cfo_insert_mt, self.fill_keys, a, s, 1)
            tn += self._run(self.L.cfo_insert_mt, self.fill_keys, a + s, b - a - s, self.threads)
            n1 += s
            nn += b - a - s
        self.rates["insert"] = {1: n1 / t1, self.threads: nn / tn}
        self.fill_seconds = t1 + tn
        self.load = self.o.occupied() / float(self.o.nb * self.o.bucket_size)

    def step(self, k: int) -> dict:
        nq, nd = len(self.query), len(self.dele)
        qa = (k * self.q_slice) % max(1, nq - self.q_slice + 1)
        da = (k * self.d_slice) % max(1, nd - self.d_slice + 1)
        q1, d1 = max(1, self.q_slice // 16), max(1, self.d_slice // 16)
        r = {"contains": {}, "delete": {}}
        L = self.L
        r["contains"][self.threads] = self.q_slice / self._run(L.cfo_contains_mt, self.query, qa, self.q_slice,
                                                               self.threads)
        r["contains"][1] = q1 / self._run(L.cfo_contains_mt, self.query, qa, q1, 1)
        r["delete"][self.threads] = self.d_slice / self._run(L.cfo_delete_mt, self.dele, da, self.d_slice,
                                                             self.threads)
        self._run(L.cfo_insert_mt, self.dele, da, self.d_slice, self.threads)
        r["delete"][1] = d1 / self._run(L.cfo_delete_mt, self.dele, da, d1, 1)
        self._run(L.cfo_insert_mt, self.dele, da, d1, self.threads)
        out = {}
        for t in (1, self.threads):
            secs = (self.n[0] / self.rates["insert"][t] + self.n[1] / r["contains"][t]
                    + self.n[2] / r["delete"][t])
            out[t] = {"value": sum(self.n) / secs / 1e9, "seconds_per_step": secs,
                      "insert_gkeys_s": self.rates["insert"][t] / 1e9,
                      "contains_gkeys_s": r["contains"][t] / 1e9, "delete_gkeys_s": r["delete"][t] / 1e9}
        return out

    def describe(self) -> str:
        return (f"full-size {self.o.nb * self.o.bucket_size}-slot table (oracle/cf_oracle.c port of the reference "
                f"algorithm): one fill of all {self.n[0]} keys in {self.STRATA} load strata (1/{self.ONE_IN} of each "
                f"stratum by one thread, the rest by {self.threads}), reaching load {self.load:.4f}; per step at that "
                f"load, {self.q_slice} lookups and {self.d_slice} deletes by {self.threads} threads and 1/16 of each "
                f"by one thread; the step's rate is the workload's mix ({self.n[0]} inserts, {self.n[1]} lookups, "
                f"{self.n[2]} deletes) at the measured per-op rates")


def cpu_baseline_entry(tab: "CpuFullTable", per_step: list) -> dict:
    """cpu_baseline object: the all-threads figure as `value`, and both thread counts."""
    th = tab.threads
    entries = {}
    for t in (1, th):
        v = [s[t] for s in per_step]
        entries[f"threads_{t}"] = {k: statistics.mean(x[k] for x in v) for k in v[0]}
    return {"value": entries[f"threads_{th}"]["value"], "unit": "Gkeys/s", "cores": th, "kind": "port",
            "sample": tab.describe(), "cpu_model": cpu_model(), "fill_seconds": tab.fill_seconds,
            "threads": {"1": entries["threads_1"], str(th): entries[f"threads_{th}"]}}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def workload_config(args, w: dict, world: int) -> dict:
    """The `config` object of the plain form's JSON line: the workload alone,
    identical in the library's arm and the reference arm."""
    import oracle

    cap, bs, bits = w["capacity"], w["bs"], w["bits"]
    nb = oracle.num_buckets(cap, bs)
    n_fill = int(w["fill"] * cap)
    sorted_fill = args.insert == "sorted" or (args.insert == "auto" and n_fill >= (1 << 29))
    return {"workload": args.workload, "desc": w["desc"], "capacity_slots": cap, "num_buckets": nb,
            "table_bytes": nb * bs * bits // 8, "bits_per_tag": bits, "bucket_size": bs, "eviction": w["policy"],
            "max_evictions": w["max_ev"], "block_size": args.block,
            "insert_path": "insertManySorted" if sorted_fill else "insertMany",
            "fill_keys": n_fill, "lookup_keys": w["n_pos"] + w["n_neg"], "delete_keys": w["n_del"],
            "l2": "inputs larger than L2 (table and key arrays exceed 126 MB); no flush needed"
            if cap >= (1 << 26) else "table L2-resident (small workload)",
            "parallelism": f"{world} independent filter shard(s), one per GPU, no collective"}


# ------------------------------------------------------------ GPU benchmark


def run_b200(args, w: dict) -> dict | None:
    import torch

    from __graft_entry__ import package

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfb = package()
    stream = torch.cuda.current_stream()

    cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=w["bits"], maxEvictions=w["max_ev"], blockSize=args.block,
                           bucketSize=w["bs"], evictionPolicy=cfb.EvictionPolicy[w["policy"]])
    f = cfb.CuckooFilter(cfg, w["capacity"])
    if args.workspace_gb is not None:
        f.setOption(cfb.OPT_WORKSPACE_LIMIT, int(args.workspace_gb * (1 << 30)))
    staging = {"auto": cfb.STAGING_AUTO, "random": cfb.STAGING_RANDOM, "segment": cfb.STAGING_SEGMENT,
               "region": cfb.STAGING_REGION}[args.staging]
    f.setOption(cfb.OPT_STAGING, staging)
    fill, query, dele, n_coll, is_pos = make_inputs(w, dev, rank, with_mask=True)
    n_fill, n_q, n_d = fill.numel(), query.numel(), dele.numel()
    q_out = torch.empty(n_q, dtype=torch.bool, device=dev)
    torch.cuda.synchronize()
    # the reference benchmark's adaptiveInsert (benchmark_common.cuh:113-126): sorted from 2^29 keys
    sorted_fill = args.insert == "sorted" or (args.insert == "auto" and n_fill >= (1 << 29))

    def fill_table(sync: bool):
        if sorted_fill:
            f.insertManySorted(fill, stream=stream)
        elif sync:
            f.insertMany(fill, stream=stream)
        else:
            f.insertManyAsync(fill, stream=stream)

    def step(ev=None):
        if ev:
            ev[0].record(stream)
        f.clear(stream)  # synchronous memset of the table and counters
        if ev:
            ev[1].record(stream)
        fill_table(False)
        if ev:
            ev[2].record(stream)
        f.containsManyAsync(query, q_out, stream=stream)
        if ev:
            ev[3].record(stream)
        f.deleteManyAsync(dele, stream=stream)
        if ev:
            ev[4].record(stream)

    # warm-up; the first warm-up step also yields the exact sector accounting.
    # That step fills in the reference's primary-first order (no first-round
    # cap), so `i1_full` counts the keys whose primary bucket was really full,
    # not the ones the capped first round sends on by choice.
    acct = {}
    for i in range(args.warmup):
        f.clear(stream)
        f.resetEvictionCount()
        f.setOption(cfb.OPT_ROUND1_CAP, w["bs"] if i == 0 else 0)
        fill_table(True)
        f.setOption(cfb.OPT_ROUND1_CAP, 0)
        st = f.stats()
        if i == 0:
            acct["i1_full"] = st["secondary"] + st["evicted_inserts"]
            acct["inserted"] = st["occupied"]
            acct["failed"] = st["failed"]
            acct["evictions"] = st["evictions"]
            acct["fill_stats"] = st
            acct["q_primary"] = f.probe_count(query, stream=stream)
            acct["d_primary"] = f.probe_count(dele, stream=stream)
        f.containsManyAsync(query, q_out, stream=stream)
        f.deleteMany(dele, stream=stream)
        if i == 0:
            acct["removed"] = f.stats()["removed"]
            acct["q_hits"] = int(q_out.sum().item())
    torch.cuda.synchronize()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    launches0 = cfb.launch_count()
    with ClockSampler(local) as clk:
        t_wall0 = time.perf_counter()
        for k in range(args.steps):
            step(evs[k])
        torch.cuda.synchronize()
        t_wall1 = time.perf_counter()
    launches = cfb.launch_count() - launches0
    barrier(world)
    step_ms = [evs[k][0].elapsed_time(evs[k][4]) for k in range(args.steps)]
    ins_ms = [evs[k][1].elapsed_time(evs[k][2]) for k in range(args.steps)]
    con_ms = [evs[k][2].elapsed_time(evs[k][3]) for k in range(args.steps)]
    del_ms = [evs[k][3].elapsed_time(evs[k][4]) for k in range(args.steps)]
    total_ms = sum(step_ms)
    keys_per_step = n_fill + n_q + n_d
    value, total_ms_max = aggregate(world, keys_per_step, args.steps, total_ms)
    all_keys = value * 1e9 * total_ms_max / 1e3

    peak, peak_src = measured_peak()
    ins_bytes = n_fill * (8 + 32 + 32) + 32 * acct["i1_full"]
    con_bytes = n_q * (8 + 1) + 32 * (2 * n_q - acct["q_primary"])
    del_bytes = n_d * (8 + 1) + 32 * (2 * n_d - acct["d_primary"]) + 32 * acct["removed"]

    def op(n, ms, b):
        t = statistics.mean(ms) / 1e3
        return {"gkeys_s": n / t / 1e9, "ms": statistics.mean(ms), "algorithmic_bytes": b,
                "achieved_gbs": b / t / 1e9, "frac_of_hbm": b / t / 1e9 / peak}

    ops = {"insert": {**op(n_fill, ins_ms, ins_bytes), "ms_steps": ins_ms},
           "contains": {**op(n_q, con_ms, con_bytes), "ms_steps": con_ms},
           "delete": {**op(n_d, del_ms, del_bytes), "ms_steps": del_ms}, "clear_ms": statistics.mean(
               [evs[k][0].elapsed_time(evs[k][1]) for k in range(args.steps)])}
    # the library's automatic choice (CF_OPT_SEGMENTED_MIN_KEYS = 0): inserts are
    # segment-staged from one key per bucket, lookups and deletes from eight
    def path_of(n, per_bucket):
        if args.staging != "auto":
            return {"random": "random probes", "segment": "segment-staged", "region": "region-staged"}[args.staging]
        return "segment-staged" if n >= f.getNumBuckets() * per_bucket else "random probes"

    ins_path = path_of(n_fill, 1)
    ops["insert"]["path"] = ("insertManySorted (segment-staged)" if sorted_fill and args.staging != "region" else
                             "insertManySorted (region-staged)" if sorted_fill else
                             "insertMany (random CAS)" if ins_path == "random probes" else f"insertMany ({ins_path})")
    ops["contains"]["path"] = path_of(n_q, 8)
    ops["delete"]["path"] = path_of(n_d, 8)

    # plain insertMany on the random CAS path (a fill this large would be
    # segment-staged by default), on the same fill, timed on its own
    if sorted_fill and not args.no_plain:
        f.setOption(cfb.OPT_STAGING, cfb.STAGING_RANDOM)
        ts = []
        for _ in range(max(1, min(args.steps, 3))):
            f.clear(stream)
            f.resetEvictionCount()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            f.insertManyAsync(fill, stream=stream)
            b.record(stream)
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        st_p = f.stats()
        ops["insert_plain"] = op(n_fill, ts, n_fill * 72 + 32 * (st_p["secondary"] + st_p["evicted_inserts"]))
        ops["insert_plain"]["path"] = "insertMany (random CAS), not part of the step"
        ops["insert_plain"]["failed"] = st_p["failed"]
        f.setOption(cfb.OPT_STAGING, staging)
    for name in ("insert", "contains", "delete"):
        tr = load_traffic(name, w, ops[name]["path"])
        if tr:
            ops[name]["dram_bytes"] = tr["bytes_per_launch"]
            ops[name]["dram_gbs"] = tr["bytes_per_launch"] / (ops[name]["ms"] / 1e3) / 1e9
            ops[name]["dram_frac"] = ops[name]["dram_gbs"] / peak
    dom = max(("insert", "contains", "delete"), key=lambda k: ops[k]["ms"])
    traffic = load_traffic(dom, w, ops[dom]["path"])
    # a "launch" of the dominant operation is one C-ABI call, which issues the
    # kernels listed in the committed launch-list summary under profiles/
    roof = {"bound": "hbm", "kernel": f"{dom}: {ops[dom]['path']} (one C-ABI call; kernels and shares in profiles/)",
            "achieved": ops[dom]["achieved_gbs"], "peak": peak, "unit": "GB/s",
            "frac": ops[dom]["achieved_gbs"] / peak, "peak_source": peak_src,
            "traffic": traffic.get("bytes_per_launch") if traffic else None,
            "traffic_source": traffic.get("source") if traffic else None,
            "dram_achieved": ops[dom].get("dram_gbs"), "dram_frac": ops[dom].get("dram_frac")}

    # ------------------------------------- per-key parity of the timed configuration
    if not args.no_verify:
        acct["parity"] = verify_parity(f, w, fill, query, is_pos, dele, sorted_fill, stream)
    del is_pos

    # ------------------------------------------------ end to end (host buffers)
    e2e = None
    if not args.no_e2e:
        h_fill = pinned_empty(n_fill, torch.int64)
        h_query = pinned_empty(n_q, torch.int64)
        h_del = pinned_empty(n_d, torch.int64)
        h_out = pinned_empty(n_q, torch.bool)
        h_fill.copy_(fill)
        h_query.copy_(query)
        h_del.copy_(dele)
        d_fill = torch.empty_like(fill)
        d_query = torch.empty_like(query)
        d_del = torch.empty_like(dele)
        torch.cuda.synchronize()
        n_e2e = max(1, min(args.steps, args.e2e_steps))
        copy = torch.cuda.Stream(device=dev)
        nchunk = max(1, args.e2e_chunks)
        bounds = [(n_fill * i // nchunk, n_fill * (i + 1) // nchunk) for i in range(nchunk)]
        times = []
        for k in range(n_e2e + 1):
            barrier(world)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            f.clear(stream)
            # every host->device copy is queued on a copy stream up front; each
            # synchronous C-ABI call waits only for the copy of its own input, so
            # PCIe transfers overlap the inserts of earlier chunks
            fill_ev = []
            with torch.cuda.stream(copy):
                for a, b in bounds:
                    d_fill[a:b].copy_(h_fill[a:b], non_blocking=True)
                    e = torch.cuda.Event()
                    e.record(copy)
                    fill_ev.append(e)
                d_query.copy_(h_query, non_blocking=True)
                eq = torch.cuda.Event()
                eq.record(copy)
                d_del.copy_(h_del, non_blocking=True)
                ed = torch.cuda.Event()
                ed.record(copy)
            for (a, b), e in zip(bounds, fill_ev):
                stream.wait_event(e)
                if sorted_fill:
                    f.insertManySorted(d_fill[a:b], stream=stream)
                else:
                    f.insertMany(d_fill[a:b], stream=stream)
            stream.wait_event(eq)
            f.containsMany(d_query, q_out, stream=stream)
            copy.wait_stream(stream)
            with torch.cuda.stream(copy):
                h_out.copy_(q_out, non_blocking=True)
            stream.wait_event(ed)
            f.deleteMany(d_del, stream=stream)
            torch.cuda.synchronize()
            if k:  # first pass warms the pinned pages
                times.append(time.perf_counter() - t0)
        t = max_over_ranks(world, statistics.mean(times))
        # the PCIe ceiling: a plain copy of fill keys (2 GiB at most) from pinned
        # host memory, CUDA events on the copy stream, best of three
        nb = min(n_fill, 1 << 28)
        h2d_rates = []
        for _ in range(3):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(copy)
            with torch.cuda.stream(copy):
                d_fill[:nb].copy_(h_fill[:nb], non_blocking=True)
            ev[1].record(copy)
            ev[1].synchronize()
            h2d_rates.append(8 * nb / (ev[0].elapsed_time(ev[1]) / 1e3) / 1e9)
        h2d_copy = max(h2d_rates)
        h2d_achieved = 8 * keys_per_step / t / 1e9
        del h_fill, h_query, h_del, h_out
        release_pinned()
        e2e = {"value": all_keys / args.steps / t / 1e9, "unit": "Gkeys/s",
               "h2d_bytes_per_step": 8 * keys_per_step, "d2h_bytes_per_step": n_q + 3 * 8 * 16,
               "h2d_achieved_gbs": h2d_achieved, "h2d_copy_gbs": h2d_copy, "frac_of_h2d_copy": h2d_achieved / h2d_copy,
               "ms_per_step": t * 1e3, "steps": n_e2e,
               "path": f"synchronous C-ABI calls ({'cf_insert_sorted' if sorted_fill else 'cf_insert'} in {nchunk} "
                       "chunks, cf_contains, cf_delete); inputs copied from pinned host memory on a copy stream that "
                       "runs ahead of the calls, lookup results copied back; wall clock per step"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        tab = CpuFullTable(w, fill.cpu().numpy().view(np.uint64), query.cpu().numpy().view(np.uint64),
                           dele.cpu().numpy().view(np.uint64), host_threads())
        tab.fill()
        cpu = cpu_baseline_entry(tab, [tab.step(0)])
        del tab

    st = f.stats()
    result = None
    if rank == 0:
        result = {
            "metric": METRIC, "value": value, "unit": "Gkeys/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: splitmix64 uint64 keys (seeded), positives sampled without replacement, "
                    "negatives disjoint by construction",
            "config": workload_config(args, w, world),
            "library": {"workspace_limit": "library default (automatic)" if args.workspace_gb is None
                        else f"{args.workspace_gb} GiB (CF_OPT_WORKSPACE_LIMIT)",
                        "workspace_bytes": f.getOption(cfb.OPT_WORKSPACE_BYTES), "options": "library defaults"
                        if args.workspace_gb is None else "CF_OPT_WORKSPACE_LIMIT set"},
            "ops": ops,
            "accounting": {**acct, "load_factor": acct["inserted"] / f.capacity(), "negatives_replaced": n_coll},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "wall_s_timed": t_wall1 - t_wall0,
            "lost_tags": st["lost"],
        }
    f.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return result


def verify_parity(f, w: dict, fill, query, is_pos, dele, sorted_fill: bool, stream, chunk: int = 1 << 28) -> dict:
    """Per-key parity of the timed configuration on the full workload (untimed).

    The fill is the timed steps' own (library defaults: for a large batch the
    capped three-round segment-staged insert).  Then:
      * counters against the image: occupied == countOccupiedSlots == stored
        keys, lost == 0;
      * zero false negatives over every stored fill key;
      * the table's (bucket pair, tag) multiset equals the one the stored keys
        must leave (digests from the torch restatement of the reference's
        hashing, independent of the kernels);
      * the lookup batch: every positive hits; the false positives on the
        disjoint negatives lie within 3 sigma of the expected count (per
        negative 1 - (1 - q)^(2 * bucketSize * load), q = sum over tags of
        P(tag)^2 = (2^f + 2) / 2^(2f) since a zero fingerprint becomes 1);
      * deleteMany: every deleted key reports removed, occupancy drops by
        exactly that many, and the multiset loses exactly the deleted keys'
        entries.
    The reference prints 2 * bucketSize * load / 2^f as its false-positive
    estimate (src/main.cu:458-459); it is reported beside the bound."""
    import torch

    bits, bs = w["bits"], w["bs"]
    nb = f.getNumBuckets()
    n_fill, n_d = fill.numel(), dele.numel()
    dev = fill.device
    f.clear(stream)
    f.resetEvictionCount()
    if sorted_fill:
        f.insertManySorted(fill, stream=stream)
    else:
        f.insertMany(fill, stream=stream)
    st = f.stats()
    stored_mask = None
    if st["failed"]:
        # which keys failed: the same fill again, reporting per-key results
        f.clear(stream)
        f.resetEvictionCount()
        stored_mask = torch.empty(n_fill, dtype=torch.bool, device=dev)
        if sorted_fill:
            f.insertManySorted(fill, stream=stream, d_output=stored_mask)
        else:
            f.insertMany(fill, stream=stream, d_output=stored_mask)
        st = f.stats()
    n_stored = n_fill - st["failed"]
    occ, cnt = f.occupiedSlots(), f.countOccupiedSlots()
    hit = torch.empty(min(n_fill, chunk), dtype=torch.bool, device=dev)
    false_neg = 0
    for a in range(0, n_fill, chunk):
        m = min(chunk, n_fill - a)
        f.containsManyAsync(fill[a:a + m], hit[:m], stream=stream)
        h = hit[:m] if stored_mask is None else hit[:m] | ~stored_mask[a:a + m]
        false_neg += int((~h).sum().item())
    img = f.table_image()
    dig_table = table_digest(img, bits, bs, nb)
    del img
    dig_keys = key_digest(fill, bits, nb, valid=stored_mask)
    q_out = torch.empty(query.numel(), dtype=torch.bool, device=dev)
    f.containsMany(query, q_out, stream=stream)
    pos_missed = int((is_pos & ~q_out).sum().item())
    n_neg = int((~is_pos).sum().item())
    fp_hits = int((~is_pos & q_out).sum().item())
    load = occ / f.capacity()
    q = ((1 << bits) + 2) / float(1 << (2 * bits))
    p_fp = 1.0 - (1.0 - q) ** (2 * bs * load)
    expected = n_neg * p_fp
    sigma = math.sqrt(n_neg * p_fp * (1.0 - p_fp))
    d_out = torch.empty(n_d, dtype=torch.bool, device=dev)
    occ_after = f.deleteMany(dele, d_out, stream=stream)
    removed_reported = int(d_out.sum().item())
    st_after = f.stats()
    cnt_after = f.countOccupiedSlots()
    multiset_after = None
    if stored_mask is None:  # every deleted key was stored: its entry must be the one removed
        img = f.table_image()
        multiset_after = table_digest(img, bits, bs, nb) == digest_sub(dig_keys, key_digest(dele, bits, nb))
        del img
    res = {
        "fill": "the timed steps' fill (library defaults)",
        "stored": n_stored, "failed": st["failed"], "occupied": occ, "count_occupied_slots": cnt,
        "lost": st["lost"], "duplicates": st["duplicates"], "counters_match_image": occ == cnt == n_stored,
        "false_negatives_all_fill_keys": false_neg,
        "multiset_conserved": dig_table == dig_keys, "entries_in_table": dig_table[0],
        "lookup_positives_missed": pos_missed, "lookup_negatives": n_neg, "false_positives": fp_hits,
        "fpr": fp_hits / max(1, n_neg), "fp_expected": expected, "fp_sigma": sigma,
        "fp_within_3sigma": abs(fp_hits - expected) <= 3 * sigma,
        "fpr_reference_estimate": 2 * bs * load / float(1 << bits),
        "deleted_reported": removed_reported, "delete_keys": n_d, "removed_counter": st_after["removed"],
        "occupied_after_delete": occ_after, "count_after_delete": cnt_after,
        "delete_counts_match": removed_reported == n_d == st_after["removed"]
        and occ_after == cnt_after == occ - n_d,
        "multiset_after_delete": multiset_after,
    }
    res["all_passed"] = bool(
        res["counters_match_image"] and st["lost"] == 0 and false_neg == 0 and res["multiset_conserved"]
        and pos_missed == 0 and res["fp_within_3sigma"] and res["delete_counts_match"]
        and multiset_after is not False)
    return res


def load_traffic(op: str, w: dict, path: str) -> dict | None:
    """DRAM bytes of one C-ABI call of `op` on this workload, from the committed
    ncu summary (profiles/dram_traffic.json: bytes per key of each operation and
    execution path, captured on a smaller table of the same geometry and scaled
    here by keys processed)."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
    except (OSError, ValueError):
        return None
    e = d.get(f"{op}|{path}")
    if not e:
        return None
    n = {"insert": int(w["fill"] * w["capacity"]), "contains": w["n_pos"] + w["n_neg"], "delete": w["n_del"]}[op]
    return {"bytes_per_launch": e["bytes_per_key"] * n, "source": e.get("source", p)}


# ------------------------------------------------------------ batched form


def splitmix64_segments(seeds, counts, first, device):
    """Concatenation over i of splitmix64(seeds[i]) outputs first[i] ..
    first[i] + counts[i] - 1, as one int64 tensor (one vectorised pass)."""
    import torch

    seeds_t = torch.as_tensor(seeds, dtype=torch.int64, device=device)
    counts_t = torch.as_tensor(counts, dtype=torch.int64, device=device)
    first_t = torch.as_tensor(first, dtype=torch.int64, device=device)
    seg = torch.repeat_interleave(torch.arange(len(counts), device=device), counts_t)
    starts = torch.cumsum(counts_t, 0) - counts_t
    pos = torch.arange(int(counts_t.sum().item()), device=device, dtype=torch.int64) - starts[seg] + first_t[seg]

    def lsr(z, sh):
        return (z >> sh) & ((1 << (64 - sh)) - 1)

    z = (pos + 1) * s64(G) + seeds_t[seg]
    z = (z ^ lsr(z, 30)) * s64(M1)
    z = (z ^ lsr(z, 27)) * s64(M2)
    return z ^ lsr(z, 31)


def run_batched(args) -> dict:
    """Batched form: 4096 filters with capacities log-uniform in 2^10..2^22
    slots (16-bit tags, 16-slot buckets), key batches lognormal(ln 20000, 1.5)
    clipped to 0.9 of capacity, keys splitmix64(seed = filter id).  All inserts
    in one launch, then all lookups (50 % positive) replayed from a captured
    CUDA graph; against a loop of per-filter insertMany / containsMany calls."""
    import numpy as np
    import torch

    from __graft_entry__ import package

    cfb = package()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(args.batched_seed)
    nf = args.filters
    caps = np.exp2(rng.uniform(10, 22, nf)).astype(np.uint64)
    sizes = np.minimum(rng.lognormal(np.log(20000), 1.5, nf), 0.9 * caps).astype(np.int64)
    ids = np.arange(nf, dtype=np.int64)
    keys = splitmix64_segments(ids, sizes, np.zeros(nf, np.int64), dev)
    offs = torch.zeros(nf + 1, dtype=torch.int64, device=dev)
    offs[1:] = torch.cumsum(torch.as_tensor(sizes, device=dev), 0)
    filt = torch.arange(nf, dtype=torch.int32, device=dev)
    # lookups: per filter, the first half of its batch (positives) + as many keys of another stream
    npos = sizes // 2
    nneg = sizes - npos
    pos = splitmix64_segments(ids, npos, np.zeros(nf, np.int64), dev)
    neg = splitmix64_segments(ids + (1 << 40), nneg, np.zeros(nf, np.int64), dev)
    qs = torch.cat([torch.cat([p, q]) for p, q in zip(pos.split(npos.tolist()), neg.split(nneg.tolist()))])
    qoffs = offs  # same sizes per filter
    n_keys, n_q = int(sizes.sum()), int(sizes.sum())
    q_out = torch.empty(n_q, dtype=torch.uint8, device=dev)
    cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=16, bucketSize=16, maxEvictions=500,
                           evictionPolicy=cfb.EvictionPolicy.BFS)
    stream = torch.cuda.Stream(device=dev)
    s = cfb.CuckooFilterSet(cfg, caps)
    # autotune inserts (clears the set), then fill and autotune lookups on the filled set
    t_ins_tune = s.autotune(cfb.SET_INSERT, keys, offs, filt, stream=stream)
    s.insert_async(keys, offs, filt, stream=stream)
    s.sync(stream=stream)
    t_con_tune = s.autotune(cfb.SET_CONTAINS, qs, qoffs, filt, q_out, stream=stream)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        s.contains_async(qs, qoffs, filt, q_out, stream=stream)
    torch.cuda.synchronize()
    ins_ms, con_ms = [], []
    for k in range(args.warmup + args.steps):
        s.clear(stream=stream)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        s.insert_async(keys, offs, filt, stream=stream)
        e[1].record(stream)
        with torch.cuda.stream(stream):  # replay on the stream the events are recorded on
            g.replay()
        e[2].record(stream)
        s.sync(stream=stream)
        if k >= args.warmup:
            ins_ms.append(e[0].elapsed_time(e[1]))
            con_ms.append(e[1].elapsed_time(e[2]))
    occ = s.occupied()
    set_hits = int(q_out.sum().item())
    pos_found = all(bool(q_out[int(o):int(o) + int(p)].all().item()) for o, p in
                    zip(offs[:-1].tolist()[:64], npos[:64]))  # spot check of the first 64 filters
    # baseline: a loop of per-filter calls of the plain API (synchronous, as the reference's API is)
    filters = [cfb.CuckooFilter(cfg, int(c)) for c in caps]
    kh = keys.split(sizes.tolist())
    qh = qs.split(sizes.tolist())
    outs = q_out.split(sizes.tolist())
    loop_ins, loop_con = [], []
    for k in range(max(1, min(args.steps, 2)) + 1):
        for f in filters:
            f.clear(stream)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for f, kk in zip(filters, kh):
            f.insertMany(kk, stream=stream)
        t1 = time.perf_counter()
        for f, qq, oo in zip(filters, qh, outs):
            f.containsMany(qq, oo, stream=stream)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if k:
            loop_ins.append(t1 - t0)
            loop_con.append(t2 - t1)
    loop_hits = int(q_out.sum().item())
    ti, tc = statistics.mean(ins_ms) / 1e3, statistics.mean(con_ms) / 1e3
    li, lc = statistics.mean(loop_ins), statistics.mean(loop_con)
    res = {
        "form": "batched", "metric": "Gkeys/s aggregate insert + lookup over 4096 uneven filters",
        "value": (n_keys + n_q) / (ti + tc) / 1e9, "unit": "Gkeys/s", "higher_is_better": True, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "dtype": "u64", "data": "synthetic: splitmix64(seed = filter id)",
        "config": {"workload": "batched: 4096 filters, capacities log-uniform 2^10..2^22 slots, 16/16, BFS; batches "
                               "lognormal(ln 20000, 1.5) clipped to 0.9 capacity; lookups 50% positive",
                   "filters": nf, "insert_keys": n_keys, "lookup_keys": n_q,
                   "table_bytes": int(sum(n * 32 for n in s.num_buckets))},
        "set": {"insert_gkeys_s": n_keys / ti / 1e9, "insert_ms": ti * 1e3, "lookup_gkeys_s": n_q / tc / 1e9,
                "lookup_ms": tc * 1e3, "launches_per_step": 2, "insert_launch": s.get_launch(cfb.SET_INSERT),
                "lookup_launch": s.get_launch(cfb.SET_CONTAINS), "tune_best_ms": {"insert": t_ins_tune,
                                                                                 "lookup": t_con_tune},
                "lookup_path": "one CUDA-graph replay", "hits": set_hits, "occupied": int(occ.sum()),
                "positives_found_spot_check": pos_found},
        "loop_baseline": {"insert_gkeys_s": n_keys / li / 1e9, "insert_ms": li * 1e3,
                          "lookup_gkeys_s": n_q / lc / 1e9, "lookup_ms": lc * 1e3,
                          "value": (n_keys + n_q) / (li + lc) / 1e9, "hits": loop_hits,
                          "path": "4096 synchronous insertMany calls, then 4096 containsMany calls; wall clock"},
        "speedup_vs_loop": (li + lc) / (ti + tc),
    }
    del g
    for f in filters:
        f.close()
    s.close()
    return res


# ------------------------------------------------------------- served form


def run_served(args) -> dict:
    """Served form: 256 tenant filters (capacities log-uniform 2^16..2^26
    slots, 8- or 16-bit tags) admitted under a 120 GB HBM budget; Poisson
    request arrivals at each offered load; 60/30/10 lookup/insert/delete;
    request sizes lognormal (median 16K keys, clipped 1K..1M).  Continuous
    batching over filter sets against a FIFO of plain per-request API calls."""
    import torch

    from __graft_entry__ import package

    cfb = package()
    import cuckoo_b200.serving as srv

    torch.cuda.set_device(0)
    tenants = srv.make_tenants(args.tenants, seed=args.batched_seed)
    loads = [float(x) for x in args.loads.split(",")]
    out = {"form": "served", "metric": "p50/p99 request latency and sustained Mkeys/s vs offered load",
           "unit": "ms / Mkeys/s", "n_gpus": 1, "dtype": "u64",
           "data": "synthetic: per-tenant splitmix64 streams, Poisson arrivals",
           "config": {"workload": "served: 256 tenants, capacities log-uniform 2^16..2^26 slots, 8/16-bit tags, "
                                  "16-slot buckets; 60/30/10 lookup/insert/delete; sizes lognormal(median 16384, "
                                  "sigma 1) clipped 1K..1M", "tenants": args.tenants,
                      "hbm_budget_gb": args.budget_gb, "duration_s_per_load": args.duration}, "loads": []}
    for i, load in enumerate(loads):
        trace = srv.make_trace(tenants, load * 1e6, args.duration, seed=100 + i)
        server = srv.Server(cfb, tenants, hbm_budget_bytes=int(args.budget_gb * 1e9), max_wave_keys=1 << 24)
        try:
            server.warm_up()
            served = server.run(trace)
            waves, launches = server.waves, server.launches
            admitted = len(server.admitted)
        finally:
            server.close()
        st = srv.latency_stats(served)
        import copy

        plain = srv.serve_plain(cfb, tenants, [copy.copy(r) for r in trace])
        sp = srv.latency_stats(plain)
        same = all(np.array_equal(a.result, b.result) for a, b in zip(served, plain))
        out["loads"].append({"offered_mkeys_s": load, "requests": st["requests"], "keys": st["keys"],
                             "served": {**st, "waves": waves, "kernel_launches": launches, "admitted": admitted},
                             "plain_fifo": sp, "results_identical": same})
    return out


# ------------------------------------------------------------ k-mer workload


def markov_dna(n_bases: int, chains: int, seed: int, device):
    """A DNA string (uint8 bases A=0 C=1 G=2 T=3) from an order-3 Markov chain
    whose 64 transition rows are seeded Dirichlet(1) draws (Exp(1) normalised).
    `chains` independent chains run in parallel and are concatenated."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    rows = -torch.log(torch.rand(64, 4, generator=g, device=device, dtype=torch.float64))  # Exp(1)
    rows = rows / rows.sum(1, keepdim=True)
    cum = torch.cumsum(rows, 1)[:, :3].float()  # 3 thresholds per context
    steps = n_bases // chains
    seq = torch.empty(chains, steps, dtype=torch.uint8, device=device)
    state = torch.randint(0, 64, (chains,), generator=g, device=device)
    for t in range(steps):
        u = torch.rand(chains, generator=g, device=device)
        c = cum[state]
        base = (u > c[:, 0]).to(torch.int64) + (u > c[:, 1]) + (u > c[:, 2])
        seq[:, t] = base.to(torch.uint8)
        state = ((state << 2) | base) & 63
    return seq.reshape(-1)


def mutate(bases, rate: float, seed: int):
    """Copy of `bases` with each base substituted by a different one with probability `rate`."""
    import torch

    g = torch.Generator(device=bases.device)
    g.manual_seed(seed)
    hit = torch.rand(bases.numel(), generator=g, device=bases.device) < rate
    shift = torch.randint(1, 4, (bases.numel(),), generator=g, device=bases.device, dtype=torch.uint8)
    return torch.where(hit, (bases + shift) % 4, bases)


def canonical_kmers(bases, k: int = 31):
    """Canonical k-mers (min of the 2-bit MSB-first forward encoding and its
    reverse complement) of every window, as int64."""
    import torch

    n = bases.numel() - k + 1
    b = bases.to(torch.int64)
    fwd = torch.zeros(n, dtype=torch.int64, device=bases.device)
    rc = torch.zeros(n, dtype=torch.int64, device=bases.device)
    for j in range(k):
        w = b[j:j + n]
        fwd |= w << (2 * (k - 1 - j))
        rc |= (3 - w) << (2 * j)
    return torch.minimum(fwd, rc)


def run_kmer(args) -> dict:
    """Synthetic k-mer workload: a 2^28-base order-3 Markov DNA string, its
    distinct canonical 31-mers inserted in 20 equal steps up to 0.95 load
    (or as far as the distinct k-mers go), insert Gkeys/s and eviction-chain
    histogram per step; then lookups of the 31-mers of a copy with 1 % random
    substitutions."""
    import torch

    from __graft_entry__ import package

    cfb = package()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n_bases = 1 << args.kmer_bases_log2
    t0 = time.perf_counter()
    g = torch.Generator(device=dev)
    g.manual_seed(args.batched_seed + 1)
    if args.kmer_file:
        # a real k-mer set in the reference's binary format: inserted in a seeded
        # shuffle; queries are every k-mer of the set (positives) plus as many
        # splitmix64 keys (negatives up to the false-positive rate)
        from cuckoo_b200.kmer import read_kmer_file

        host = read_kmer_file(args.kmer_file)
        kmers = torch.unique(torch.from_numpy(host.view(np.int64)).to(dev))
        kmers = kmers[torch.randperm(kmers.numel(), generator=g, device=dev)]
        neg = splitmix64_segments(np.array([args.batched_seed + 3], np.int64), np.array([kmers.numel()], np.int64),
                                  np.array([0], np.int64), dev)
        queries = torch.cat([kmers, neg])
        data = f"k-mer file {os.path.basename(args.kmer_file)} ({host.size} k-mers); queries: the set plus as many splitmix64 keys"
        n_bases = 0
    else:
        dna = markov_dna(n_bases, 1 << 14, args.batched_seed, dev)
        kmers = torch.unique(canonical_kmers(dna))
        kmers = kmers[torch.randperm(kmers.numel(), generator=g, device=dev)]
        queries = canonical_kmers(mutate(dna, 0.01, args.batched_seed + 2))
        data = (f"synthetic: 2^{args.kmer_bases_log2}-base order-3 Markov DNA (Dirichlet(1) rows), canonical "
                "31-mers 2-bit MSB-first, deduplicated; queries from a 1%-substituted copy")
    gen_s = time.perf_counter() - t0
    out = {"form": "kmer", "metric": "insert Gkeys/s per load step; lookup Gkeys/s and hit rate",
           "unit": "Gkeys/s", "n_gpus": 1, "dtype": "u64", "data": data,
           "config": {"workload": "kmer", "bases": n_bases, "distinct_kmers": int(kmers.numel()),
                      "query_windows": int(queries.numel()), "generation_s": gen_s}, "filters": []}
    stream = torch.cuda.current_stream()
    for cap_log2, bits in ((26, 8), (30, 16)):
        cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=bits, bucketSize=16, maxEvictions=500,
                               evictionPolicy=cfb.EvictionPolicy.BFS)
        f = cfb.CuckooFilter(cfg, 1 << cap_log2)
        f.setOption(cfb.OPT_CHAIN_HISTOGRAM, 1)
        target = int(0.95 * f.capacity())
        n_ins = min(target, kmers.numel())
        per = n_ins // 20
        steps = []
        prev_hist = np.zeros(10, np.uint64)
        for st_i in range(20):
            a = st_i * per
            b = n_ins if st_i == 19 else a + per
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            occ = f.insertMany(kmers[a:b], stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            hist = f.chainHistogram()
            stt = f.stats()
            steps.append({"step": st_i + 1, "keys": b - a, "load": occ / f.capacity(), "ms": ms,
                          "insert_gkeys_s": (b - a) / ms / 1e6, "failed_total": stt["failed"],
                          "chain_histogram": (hist - prev_hist).tolist()})
            prev_hist = hist
        q_out = torch.empty(queries.numel(), dtype=torch.bool, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f.containsManyAsync(queries, q_out, stream=stream)  # warm-up
        e0.record(stream)
        f.containsManyAsync(queries, q_out, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out["filters"].append({
            "capacity_slots": f.capacity(), "bits_per_tag": bits, "table_bytes": f.sizeInBytes(),
            "l2_resident": f.sizeInBytes() <= (126 << 20), "inserted": n_ins, "final_load": f.loadFactor(),
            "reached_target_load": n_ins == target,
            "chain_bins": "0 moves, 1, 2-3, 4-7, 8-15, 16-31, 32-63, 64-127, 128-255, >=256",
            "steps": steps, "lookup": {"keys": int(queries.numel()), "ms": ms,
                                       "gkeys_s": queries.numel() / ms / 1e6,
                                       "hit_rate": float(q_out.float().mean().item())}})
        f.close()
    return out


# ------------------------------------------------------------- config grid


def run_grid(args) -> dict:
    """The large filter across tag/bucket geometries, eviction policies and
    insert paths: 2^31 slots, {8/16, 16/16, 32/8} x {BFS, DFS} x {insertMany,
    insertManySorted}; fill to 0.95, 2^28 lookups (50 % positive), 2^26 deletes."""
    import torch

    from __graft_entry__ import package

    cfb = package()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    base = dict(WORKLOADS["large"])
    fill, query, dele, _ = make_inputs(base, dev)
    q_out = torch.empty(query.numel(), dtype=torch.bool, device=dev)
    stream = torch.cuda.current_stream()
    rows = []
    for bits, bs in ((8, 16), (16, 16), (32, 8)):
        for pol in ("BFS", "DFS"):
            cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=bits, bucketSize=bs, maxEvictions=500,
                                   evictionPolicy=cfb.EvictionPolicy[pol])
            f = cfb.CuckooFilter(cfg, base["capacity"])
            if args.workspace_gb is not None:
                f.setOption(cfb.OPT_WORKSPACE_LIMIT, int(args.workspace_gb * (1 << 30)))
            for path in ("insertMany", "insertManySorted"):
                res = {}
                for k in range(2):  # the first pass warms the workspace and the caches
                    f.clear(stream)
                    f.resetEvictionCount()
                    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
                    # insertMany rows: the random CAS path (the default would stage this fill)
                    f.setOption(cfb.OPT_STAGING, cfb.STAGING_RANDOM if path == "insertMany" else cfb.STAGING_AUTO)
                    e[0].record(stream)
                    if path == "insertMany":
                        f.insertManyAsync(fill, stream=stream)
                    else:
                        f.insertManySorted(fill, stream=stream)
                    e[1].record(stream)
                    f.setOption(cfb.OPT_STAGING, cfb.STAGING_AUTO)
                    f.containsManyAsync(query, q_out, stream=stream)
                    e[2].record(stream)
                    f.deleteManyAsync(dele, stream=stream)
                    e[3].record(stream)
                    torch.cuda.synchronize()
                    st = f.stats()
                    res = {"geometry": f"{bits}/{bs}", "eviction": pol, "insert_path": path,
                           "table_bytes": f.sizeInBytes(),
                           "insert_gkeys_s": fill.numel() / e[0].elapsed_time(e[1]) / 1e6,
                           "lookup_gkeys_s": query.numel() / e[1].elapsed_time(e[2]) / 1e6,
                           "delete_gkeys_s": dele.numel() / e[2].elapsed_time(e[3]) / 1e6,
                           "failed": st["failed"], "lost": st["lost"], "evictions": st["evictions"],
                           "lookup_hits": int(q_out.sum().item())}
                rows.append(res)
                print(json.dumps(res), file=sys.stderr, flush=True)
            f.close()
    return {"form": "grid", "metric": "Gkeys/s per op across geometries, eviction policies and insert paths",
            "unit": "Gkeys/s", "n_gpus": 1, "dtype": "u64", "data": "synthetic: splitmix64 keys (large workload)",
            "config": {"workload": "large filter grid: 2^31 slots; fill 0.95 (2 040 109 465 keys), 2^28 lookups "
                                   "50% positive, 2^26 deletes"}, "rows": rows}


# ------------------------------------------------------- alternate-bucket policies


def _time_fill_query_delete(cfb, f, path, fill, query, dele, q_out, stream) -> dict:
    """One cleared fill (insertMany on the random CAS path, or
    insertManySorted), lookups and deletes, each timed with CUDA events on
    `stream`."""
    import torch

    f.clear(stream)
    f.resetEvictionCount()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    # a fill this large would be segment-staged by default: force random CAS
    f.setOption(cfb.OPT_STAGING, cfb.STAGING_RANDOM if path == "insertMany" else cfb.STAGING_AUTO)
    e[0].record(stream)
    if path == "insertMany":
        f.insertManyAsync(fill, stream=stream)
    else:
        f.insertManySorted(fill, stream=stream)
    e[1].record(stream)
    f.setOption(cfb.OPT_STAGING, cfb.STAGING_AUTO)
    f.containsManyAsync(query, q_out, stream=stream)
    e[2].record(stream)
    f.deleteManyAsync(dele, stream=stream)
    e[3].record(stream)
    torch.cuda.synchronize()
    st = f.stats()
    return {"insert_gkeys_s": fill.numel() / e[0].elapsed_time(e[1]) / 1e6,
            "lookup_gkeys_s": query.numel() / e[1].elapsed_time(e[2]) / 1e6,
            "delete_gkeys_s": dele.numel() / e[2].elapsed_time(e[3]) / 1e6,
            "failed": st["failed"], "lost": st["lost"], "evictions": st["evictions"],
            "lookup_hits": int(q_out.sum().item())}


def run_policies(args) -> dict:
    """The three alternate-bucket policies on the large workload's keys
    (the reference's bucket_policy_benchmark.cu configurations: 16-bit tags,
    16-slot buckets, DFS): 2^31 slots filled to 0.95 with insertMany and with
    insertManySorted, 2^28 lookups (50 % positive), 2^26 deletes."""
    import torch

    from __graft_entry__ import package

    cfb = package()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    base = dict(WORKLOADS["large"])
    fill, query, dele, _ = make_inputs(base, dev)
    q_out = torch.empty(query.numel(), dtype=torch.bool, device=dev)
    stream = torch.cuda.current_stream()
    rows = []
    for name in ("XorAltBucketPolicy", "AddSubAltBucketPolicy", "OffsetAltBucketPolicy"):
        cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=16, bucketSize=16, maxEvictions=500,
                               evictionPolicy=cfb.EvictionPolicy.DFS, AltBucketPolicy=name)
        f = cfb.CuckooFilter(cfg, base["capacity"])
        if args.workspace_gb is not None:
            f.setOption(cfb.OPT_WORKSPACE_LIMIT, int(args.workspace_gb * (1 << 30)))
        for path in ("insertMany", "insertManySorted"):
            res = {}
            for _ in range(2):  # the first pass warms the workspace and the caches
                res = _time_fill_query_delete(cfb, f, path, fill, query, dele, q_out, stream)
            res = {"policy": name, "insert_path": path, "num_buckets": f.getNumBuckets(),
                   "table_bytes": f.sizeInBytes(), **res}
            rows.append(res)
            print(json.dumps(res), file=sys.stderr, flush=True)
        f.close()
    return {"form": "policies", "metric": "Gkeys/s per op for each alternate-bucket policy", "unit": "Gkeys/s",
            "n_gpus": 1, "dtype": "u64", "data": "synthetic: splitmix64 keys (large workload)",
            "config": {"workload": "2^31 slots, 16/16, DFS, insertMany / insertManySorted to 0.95 (2 040 109 465 "
                                   "keys), 2^28 lookups 50% positive, 2^26 deletes"}, "rows": rows}


def sharded_step(f, fill, query, dele, marks=None) -> tuple:
    """One step of the plain workload through the hash-partitioned front end
    (CuckooFilterMultiGPU): every rank inserts its own fill keys, looks up its
    own query batch and deletes its own delete batch; keys travel to the rank
    that owns them and results come back in the caller's order.  `marks`, if
    given, is called between the phases (0 before the insert, 1, 2 and 3 after
    each phase) to record timing events.  Returns (lookup results, per-key
    delete results) aligned with `query` and `dele`."""
    if marks:
        marks(0)
    f.insertMany(fill)
    if marks:
        marks(1)
    q_out = f.containsMany(query)
    if marks:
        marks(2)
    d_out = f.torch.empty(dele.numel(), dtype=f.torch.bool, device=q_out.device)
    f.deleteMany(dele, d_out)
    if marks:
        marks(3)
    return q_out, d_out


def sharded_capacity(world: int, slots_per_rank: int) -> int:
    """Total capacity of CuckooFilterMultiGPU that gives each of `world` ranks
    a shard of `slots_per_rank` slots: the per-GPU capacity
    SDIV(capacity, N) * 1.02 (CuckooFilterMultiGPU.cuh:337) stays within one
    power-of-two bucket count."""
    return int(world * (slots_per_rank - 64) / 1.02)


def run_b200_sharded(args, w: dict) -> dict | None:
    """The plain workload on N GPUs through the hash-partitioned front end
    (cuckoo-filter_b200/multigpu.py; the reference's CuckooFilterMultiGPU,
    CuckooFilterMultiGPU.cuh:168-322): each rank brings the workload's batch
    (its own key streams, seeds offset by rank), keys are grouped on the device
    and exchanged with NCCL all-to-all, each rank's shard of the workload's
    capacity runs the batch operation, and lookup and delete results come back
    in batch order.  Weak scaling: N shards of the workload's size."""
    import torch

    from __graft_entry__ import package

    cfb = package()
    import cuckoo_b200.multigpu as mg

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    own_group = False
    import torch.distributed as dist

    if not dist.is_initialized():  # one rank without torchrun: a group of one
        import datetime
        import socket

        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", str(port))
        dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        own_group = True
    world = dist.get_world_size()
    stream = torch.cuda.current_stream()
    cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=w["bits"], maxEvictions=w["max_ev"], blockSize=args.block,
                           bucketSize=w["bs"], evictionPolicy=cfb.EvictionPolicy[w["policy"]])
    f = mg.CuckooFilterMultiGPU(cfg, sharded_capacity(world, w["capacity"]), routing=args.routing,
                                max_keys_per_call=1 << 31)
    fill, query, dele, _, is_pos = make_inputs(w, dev, rank, with_mask=True)
    n_fill, n_q, n_d = fill.numel(), query.numel(), dele.numel()
    for _ in range(args.warmup):
        f.clear()
        sharded_step(f, fill, query, dele)
    torch.cuda.synchronize()
    phases = []
    launches0 = cfb.launch_count()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            f.clear()
            barrier(world)
            torch.cuda.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            q_out, d_out = sharded_step(f, fill, query, dele, marks=lambda i: ev[i].record(stream))
            torch.cuda.synchronize()
            phases.append([ev[i].elapsed_time(ev[i + 1]) for i in range(3)])
    launches = cfb.launch_count() - launches0
    # the last step's results: every positive found, every delete removed
    pos_missed = int((is_pos & ~q_out).sum().item())
    fp = int((~is_pos & q_out).sum().item())
    removed = int(d_out.sum().item())
    st = f.ops.filter.stats()
    failed = int(_reduce(world, float(st["failed"] + st["lost"]), "sum"))
    total_ms = max_over_ranks(world, sum(sum(p) for p in phases))
    ph = [max_over_ranks(world, statistics.mean(p[i] for p in phases)) for i in range(3)]
    keys_per_step = n_fill + n_q + n_d
    all_keys = sum_over_ranks(world, keys_per_step * args.steps)
    value = all_keys / (total_ms / 1e3) / 1e9
    peak, peak_src = measured_peak()
    # the rank's own shard: inserts of the keys it received, 72 B each (no primary-full credit)
    recv = st["primary"] + st["secondary"] + st["evicted_inserts"]  # the last step's (cleared each step)
    ins_bytes = 72 * recv
    ok = sum_over_ranks(world, float(pos_missed == 0 and removed == n_d and failed == 0))
    # end to end: every step copies the rank's inputs from pinned host memory
    # into the device buffers and the lookup results back
    e2e = None
    if not args.no_e2e:
        hosts = [pinned_empty(t.numel(), t.dtype) for t in (fill, query, dele)]
        h_out = pinned_empty(n_q, torch.bool)
        for h, t in zip(hosts, (fill, query, dele)):
            h.copy_(t)
        times = []
        for k in range(max(1, min(args.steps, args.e2e_steps)) + 1):
            f.clear()
            barrier(world)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for h, t in zip(hosts, (fill, query, dele)):
                t.copy_(h, non_blocking=True)
            q_e, _ = sharded_step(f, fill, query, dele)
            h_out.copy_(q_e)
            torch.cuda.synchronize()
            if k:
                times.append(time.perf_counter() - t0)
        t = max_over_ranks(world, statistics.mean(times))
        del hosts, h_out
        release_pinned()
        e2e = {"value": all_keys / args.steps / t / 1e9, "unit": "Gkeys/s",
               "h2d_bytes_per_step": 8 * keys_per_step * world, "d2h_bytes_per_step": n_q * world,
               "ms_per_step": t * 1e3, "steps": len(times),
               "path": "CuckooFilterMultiGPU insertMany / containsMany / deleteMany on every rank; inputs copied "
                       "from pinned host memory, lookup results copied back; wall clock per step, max over ranks"}
    result = None
    if rank == 0:
        result = {
            "metric": METRIC, "value": value, "unit": "Gkeys/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: splitmix64 uint64 keys (seeded per rank), positives sampled without replacement, "
                    "negatives disjoint by construction",
            "config": {**workload_config(args, w, world),
                       "parallelism": f"{world} hash-partitioned shards of {w['capacity']} slots "
                                      f"(CuckooFilterMultiGPU, {args.routing} routing), keys and results "
                                      "exchanged with NCCL all-to-all"},
            "ops": {"insert": {"ms": ph[0], "gkeys_s": world * n_fill / ph[0] / 1e6},
                    "contains": {"ms": ph[1], "gkeys_s": world * n_q / ph[1] / 1e6},
                    "delete": {"ms": ph[2], "gkeys_s": world * n_d / ph[2] / 1e6}},
            "roofline": {"bound": "hbm", "kernel": "insert phase on rank 0's shard (grouping, exchange and "
                                                  "the shard's insertMany)",
                         "achieved": ins_bytes / (ph[0] / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": ins_bytes / (ph[0] / 1e3) / 1e9 / peak, "peak_source": peak_src,
                         "traffic": None},
            "accounting": {"ranks_all_checks_passed": int(ok), "positives_missed_rank0": pos_missed,
                           "false_positives_rank0": fp, "removed_rank0": removed, "absent_inserts_all": failed},
            "cpu_baseline": None, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary()}
    del f
    if own_group:
        dist.destroy_process_group()
    return result


def run_sharded(args) -> dict | None:
    """The hash-partitioned multi-GPU form (CuckooFilterMultiGPU: one rank per
    GPU, keys grouped on the device and exchanged with NCCL all-to-all).  The
    filter's capacity gives each rank a 2^S-slot shard (16/16, BFS; S =
    --shard-slots-log2, 28 by default); per rank and step: 0.95 * 2^S keys
    inserted, 2^(S-1) lookups (half of them the rank's own keys, half never
    inserted) and 2^(S-2) deletes; CUDA events around each
    call, max over ranks.  Also the grouping kernels alone on the rank's keys
    with 8 shards, against their algorithmic bytes (28 B per key for the
    partition, 6 B for the unpartition)."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist

    from __graft_entry__ import package

    cfb = package()
    import cuckoo_b200.multigpu as mg

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    own_group = False
    if not dist.is_initialized():
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", str(port))
        dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        own_group = True
    world = dist.get_world_size()
    peak, peak_src = measured_peak()
    slots = 1 << args.shard_slots_log2
    n = int(0.95 * slots)
    q4 = slots // 4
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    splitmix64_torch(11 + 1000 * rank, 0, n, keys)
    neg = torch.empty(q4, dtype=torch.int64, device=dev)
    splitmix64_torch(12 + 1000 * rank, 0, q4, neg)
    query = torch.cat([keys[:q4], neg])
    dele = keys[q4: 2 * q4].clone()
    stream = torch.cuda.current_stream()

    def timed(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    grp = mg.KeyGrouping(dev, 8)
    holder = {}

    def part():
        holder["p"] = grp.partition(keys, 8)

    for _ in range(args.warmup):
        part()
    part_ms = max_over_ranks(world, timed(part, args.steps))
    _, pos, _ = holder["p"]
    res = torch.randint(0, 2, (n,), dtype=torch.uint8, device=dev)
    unpart_ms = max_over_ranks(world, timed(lambda: grp.unpartition(res, pos), args.steps))
    del holder, pos, res

    # SDIV(cap, N) * 1.02 stays below `slots`: a `slots`-slot shard per rank
    cap = int(world * (slots - 64) / 1.02)
    cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=16, bucketSize=16, evictionPolicy=cfb.EvictionPolicy.BFS,
                           maxEvictions=500)
    f = mg.CuckooFilterMultiGPU(cfg, cap, routing=args.routing)
    assert f.ops.filter.capacity() == slots
    phases = {"insert": [], "lookup": [], "delete": []}
    for step in range(args.warmup + args.steps):
        f.clear()
        barrier(world)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        f.insertMany(keys)
        ev[1].record(stream)
        f.containsMany(query)
        ev[2].record(stream)
        f.deleteMany(dele)
        ev[3].record(stream)
        torch.cuda.synchronize()
        if step >= args.warmup:
            for k, (a, b) in zip(phases, ((0, 1), (1, 2), (2, 3))):
                phases[k].append(max_over_ranks(world, ev[a].elapsed_time(ev[b])))
    st = f.ops.filter.stats()
    failed = int(_reduce(world, float(st["failed"]), "sum"))
    ms = {k: statistics.median(v) for k, v in phases.items()}
    step_ms = sum(ms.values())
    keys_step = world * (n + query.numel() + dele.numel())
    out = None
    if rank == 0:
        out = {"form": "sharded", "metric": "Gkeys/s insert + lookup + delete through CuckooFilterMultiGPU",
               "value": keys_step / step_ms / 1e6, "unit": "Gkeys/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
               "dtype": "u64", "data": "synthetic: splitmix64 keys",
               "config": {"workload": f"per rank: a 2^{args.shard_slots_log2}-slot shard (16/16, BFS), 0.95 * "
                                      f"2^{args.shard_slots_log2} inserts, 2^{args.shard_slots_log2 - 1} lookups "
                                      f"(50% positive), 2^{args.shard_slots_log2 - 2} deletes",
                          "routing": args.routing},
               "ops": {k: {"ms": v, "gkeys_s": world * c / v / 1e6}
                       for (k, v), c in zip(ms.items(), (n, query.numel(), dele.numel()))},
               "failed_inserts": failed,
               "grouping": {"shards": 8, "keys": n,
                            "partition": {"ms": part_ms, "gbs": 28 * n / part_ms / 1e6,
                                          "frac": 28 * n / part_ms / 1e6 / peak},
                            "unpartition": {"ms": unpart_ms, "gbs": 6 * n / unpart_ms / 1e6,
                                            "frac": 6 * n / unpart_ms / 1e6 / peak},
                            "peak_gbs": peak, "peak_source": peak_src}}
    if own_group:
        dist.destroy_process_group()
    return out


# ------------------------------------------------------- lookup-ceiling measurements


def run_gather(args) -> dict:
    """DRAM cost of random 32-byte bucket probes, for an ncu capture of one
    launch: 2^24 keys each load their primary bucket once (k_probe_count,
    through cf_probe_count) from a 1 GiB table (2^29 slots, 16-bit tags,
    16-slot buckets: 2^25 buckets of 32 bytes).  Besides the probes the kernel
    streams only the keys (8 bytes each)."""
    import torch

    from __graft_entry__ import package

    cfb = package()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=16, bucketSize=16, evictionPolicy=cfb.EvictionPolicy.BFS)
    f = cfb.CuckooFilter(cfg, 1 << 29)
    n = 1 << 24
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    splitmix64_torch(21, 0, n, keys)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        f.probe_count(keys, stream=stream)
    ms = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        f.probe_count(keys, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    out = {"form": "gather", "metric": "random 32-byte bucket probes per second (k_probe_count)", "unit": "Gprobes/s",
           "value": n / statistics.median(ms) / 1e6, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "config": {"workload": "gather: 2^24 keys, one primary-bucket probe each, 1 GiB table (2^25 buckets "
                                  "of 32 B)", "probes": n, "table_bytes": f.sizeInBytes()},
           "ms_call_median": statistics.median(ms),
           "note": "the call includes a counter allocation and read-back; per-probe DRAM bytes come from the ncu "
                   "capture of the kernel alone"}
    f.close()
    return out


def run_lookup_paths(args, w: dict) -> dict:
    """Lookups and deletes of the workload on each execution path, on the same
    filled table: random probes (one lane per key, and every warp-cooperative
    width CF_OPT_PROBE_WIDTH the geometry supports), segment-staged and
    region-staged (CF_OPT_STAGING), CUDA events per call, with the lookup
    results required to be identical across paths and every delete to
    succeed."""
    import torch

    from __graft_entry__ import package

    cfb = package()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    cfg = cfb.CuckooConfig(T="uint64_t", bitsPerTag=w["bits"], maxEvictions=w["max_ev"], bucketSize=w["bs"],
                           evictionPolicy=cfb.EvictionPolicy[w["policy"]])
    f = cfb.CuckooFilter(cfg, w["capacity"])
    fill, query, dele, _ = make_inputs(w, dev)
    stream = torch.cuda.current_stream()
    f.insertManySorted(fill, stream=stream)
    del fill
    torch.cuda.empty_cache()
    q_out = torch.empty(query.numel(), dtype=torch.bool, device=dev)
    d_out = torch.empty(dele.numel(), dtype=torch.bool, device=dev)
    ref_out = None
    rows = []
    peak, _ = measured_peak()
    bb = w["bits"] * w["bs"] // 8
    coop = [k for k in (2, 4, 8, 16, 32) if bb % k == 0 and bb // k in (4, 8) and w["bs"] <= 64]
    paths = [("random probes", cfb.STAGING_RANDOM, 0)]
    paths += [(f"random probes, {k} lanes per key (warp-cooperative, ballot / shuffle)", cfb.STAGING_RANDOM, k)
              for k in coop]
    paths += [("segment-staged", cfb.STAGING_SEGMENT, 0), ("region-staged", cfb.STAGING_REGION, 0)]
    for name, mode, width in paths:
        f.setOption(cfb.OPT_STAGING, mode)
        f.setOption(cfb.OPT_PROBE_WIDTH, width)
        con, dl = [], []
        for k in range(args.warmup + args.steps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(stream)
            f.containsManyAsync(query, q_out, stream=stream)
            e[1].record(stream)
            f.deleteManyAsync(dele, d_out, stream=stream)
            e[2].record(stream)
            torch.cuda.synchronize()
            removed = int(d_out.sum().item())
            f.setOption(cfb.OPT_STAGING, cfb.STAGING_AUTO)
            f.setOption(cfb.OPT_PROBE_WIDTH, 0)
            f.insertMany(dele, stream=stream)  # put the deleted keys back (untimed)
            f.setOption(cfb.OPT_STAGING, mode)
            f.setOption(cfb.OPT_PROBE_WIDTH, width)
            if k >= args.warmup:
                con.append(e[0].elapsed_time(e[1]))
                dl.append(e[1].elapsed_time(e[2]))
        if ref_out is None:
            ref_out = q_out.clone()
        q_primary = f.probe_count(query, stream=stream)
        con_bytes = query.numel() * 9 + 32 * (2 * query.numel() - q_primary)
        rows.append({"path": name, "probe_width": max(width, 1), "contains_ms": statistics.median(con),
                     "contains_gkeys_s": query.numel() / statistics.median(con) / 1e6,
                     "contains_frac_sector_roofline": con_bytes / (statistics.median(con) / 1e3) / 1e9 / peak,
                     "delete_ms": statistics.median(dl), "delete_gkeys_s": dele.numel() / statistics.median(dl) / 1e6,
                     "lookups_identical_to_random": bool(torch.equal(q_out, ref_out)),
                     "deletes_all_removed": removed == dele.numel()})
        print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    f.close()
    return {"form": "lookup_paths", "metric": "lookup and delete Gkeys/s per execution path", "unit": "Gkeys/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "dtype": "u64",
            "data": "synthetic: splitmix64 keys", "config": {"workload": args.workload, "desc": w["desc"]},
            "rows": rows}


# ------------------------------------------------------------ forms summary


def run_forms_summary(args) -> dict:
    """The batched and served forms in brief, for the default bench line:
    the batched form over 1024 uneven filters (the 4096-filter workload's
    distributions; the full form is --form batched) against a loop of plain
    per-filter calls, and the served form at an offered 200 Mkeys/s for
    0.25 s of arrivals against a FIFO of plain per-request calls (the full
    sweep is --form served)."""
    import copy

    import torch

    a = copy.copy(args)
    a.filters, a.steps, a.warmup = 1024, 3, 1
    b = run_batched(a)
    torch.cuda.empty_cache()
    a = copy.copy(args)
    a.loads, a.duration = "200", 0.25
    sv = run_served(a)
    torch.cuda.empty_cache()
    ld = sv["loads"][0]
    return {
        "batched": {"workload": f"{b['config']['filters']} filters, capacities log-uniform 2^10..2^22 slots, 16/16; "
                                "batches lognormal(ln 20000, 1.5); one persistent insert launch, lookups from one "
                                "captured graph",
                    "gkeys_s": b["value"], "insert_gkeys_s": b["set"]["insert_gkeys_s"],
                    "lookup_gkeys_s": b["set"]["lookup_gkeys_s"], "plain_loop_gkeys_s": b["loop_baseline"]["value"],
                    "speedup_vs_plain_loop": b["speedup_vs_loop"],
                    "same_hits": b["set"]["hits"] == b["loop_baseline"]["hits"]},
        "served": {"workload": "256 tenants, Poisson arrivals at 200 Mkeys/s offered for 0.25 s, 60/30/10 "
                               "lookup/insert/delete",
                   "p50_ms": ld["served"]["p50_ms"], "p99_ms": ld["served"]["p99_ms"],
                   "mkeys_s": ld["served"]["throughput_mkeys_s"],
                   "plain_fifo": {"p50_ms": ld["plain_fifo"]["p50_ms"], "p99_ms": ld["plain_fifo"]["p99_ms"],
                                  "mkeys_s": ld["plain_fifo"]["throughput_mkeys_s"]},
                   "results_identical": ld["results_identical"]},
    }


# ------------------------------------------------------------ reference arm


def run_reference(args, w: dict) -> dict | None:
    """The reference arm: the reference's algorithm on the host cores (the
    oracle's port; the reference's own CPU cuckoo library is not vendored) on
    the workload's full-size table, all host threads and one thread; beside it,
    where they were built from the reference's sources, the reference's own
    CUDA kernels on the full workload on this GPU."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    import torch

    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    fill, query, dele, _ = make_inputs(w, dev)
    h = [t.cpu().numpy().view(np.uint64) for t in (fill, query, dele)]
    del fill, query, dele
    if dev.type == "cuda":
        torch.cuda.empty_cache()
    tab = CpuFullTable(w, h[0], h[1], h[2], host_threads())
    tab.fill()
    for k in range(args.warmup):
        tab.step(k)
    per_step = [tab.step(args.warmup + k) for k in range(args.steps)]
    cpu = cpu_baseline_entry(tab, per_step)
    del tab, h
    value = cpu["value"]
    th = cpu["threads"][str(cpu["cores"])]
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gkeys/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": th["seconds_per_step"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic: splitmix64 uint64 keys (seeded), positives sampled without replacement, "
                "negatives disjoint by construction",
        "config": workload_config(args, w, 1),
        "cpu_baseline": {**cpu, "sample": cpu["sample"] + " (the reference's CPU cuckoo library, "
                                                          "efficient/cuckoofilter, is not vendored; this is the "
                                                          "reference's GPU algorithm ported to host threads)"},
        "e2e": {"value": value, "unit": "Gkeys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ops": {k: th[k] for k in ("insert_gkeys_s", "contains_gkeys_s", "delete_gkeys_s")},
    }
    if not args.no_ref_gpu:
        out["reference_gpu"] = run_reference_gpu(args, w)
    return out


def run_reference_gpu(args, w: dict) -> dict:
    """The reference's own CUDA kernels (compiled from its sources for sm_100a)
    on the full workload, through its public API, timed with CUDA events."""
    try:
        import torch

        import oracle
    except ImportError as e:
        return {"unavailable": str(e)}
    if oracle.ref_gpu() is None or not torch.cuda.is_available():
        return {"unavailable": "oracle/_ref/libref_gpu.so not built or no GPU"}
    pol = oracle.POLICY_BFS if w["policy"] == "BFS" else oracle.POLICY_DFS
    try:
        ref = oracle.RefGpuFilter(8, w["bits"], w["bs"], pol, w["max_ev"], w["capacity"])
    except (KeyError, RuntimeError) as e:
        return {"unavailable": f"configuration not instantiated: {e}"}
    dev = torch.device("cuda", 0)
    fill, query, dele, _, is_pos = make_inputs(w, dev, with_mask=True)
    out = torch.empty(query.numel(), dtype=torch.uint8, device=dev)
    res = {"ins": [], "con": [], "del": []}
    occ_fill = 0
    stream = torch.cuda.current_stream()
    for k in range(args.warmup + args.steps):
        ref.clear()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record(stream)
        occ_fill = ref.insert(fill.data_ptr(), fill.numel(), stream.cuda_stream or None,
                              args.insert == "sorted" or (args.insert == "auto" and fill.numel() >= (1 << 29)))
        e[1].record(stream)
        ref.contains(query.data_ptr(), query.numel(), out.data_ptr(), stream.cuda_stream or None)
        e[2].record(stream)
        ref.delete(dele.data_ptr(), dele.numel(), None, stream.cuda_stream or None)
        e[3].record(stream)
        torch.cuda.synchronize()
        if k >= args.warmup:
            res["ins"].append(e[0].elapsed_time(e[1]))
            res["con"].append(e[1].elapsed_time(e[2]))
            res["del"].append(e[2].elapsed_time(e[3]))
    occ = ref.occupied()
    ref.close()
    hits = out.to(torch.bool)
    n_neg = int((~is_pos).sum().item())
    fp = int((hits & ~is_pos).sum().item())
    same_keys = {"failed_inserts": fill.numel() - int(occ_fill), "lookup_positives_missed":
                 int((~hits & is_pos).sum().item()), "false_positives": fp, "fpr": fp / max(1, n_neg)}
    t = {k: statistics.mean(v) for k, v in res.items()}
    n_total = fill.numel() + query.numel() + dele.numel()
    return {"value": n_total / (sum(t.values()) / 1e3) / 1e9, "unit": "Gkeys/s",
            "insert_gkeys_s": fill.numel() / t["ins"] * 1e3 / 1e9,
            "contains_gkeys_s": query.numel() / t["con"] * 1e3 / 1e9,
            "delete_gkeys_s": dele.numel() / t["del"] * 1e3 / 1e9,
            "ms": t, "occupied_after": occ, "same_keys": same_keys,
            "build": "reference include/CuckooFilter.cuh compiled with -gencode arch=compute_100a,code=sm_100a "
                     "(256-bit load path live), filter object in managed memory"}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="large")
    ap.add_argument("--bits", type=int, choices=(8, 16, 32), default=None,
                    help="override the workload's bits per tag (plain form; 32-bit tags use 8-slot buckets)")
    ap.add_argument("--staging", choices=("auto", "random", "segment", "region"), default="auto",
                    help="plain form: force every batch onto one execution path (CF_OPT_STAGING)")
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--insert", choices=("auto", "plain", "sorted"), default="auto",
                    help="fill with insertMany (plain), insertManySorted (sorted), or as the reference's benchmark "
                         "does (auto: sorted from 2^29 keys)")
    ap.add_argument("--workspace-gb", type=float, default=None,
                    help="workspace limit of the segment-staged path (CF_OPT_WORKSPACE_LIMIT); default: the "
                         "library's own (automatic) limit")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the brief batched / served forms in the default line")
    ap.add_argument("--no-verify", action="store_true",
                    help="skip the untimed per-key parity check of the timed configuration")
    ap.add_argument("--no-plain", action="store_true", help="skip the separate plain insertMany timing")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--e2e-chunks", type=int, default=4, help="fill chunks of the end-to-end leg (copy/compute overlap)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--kmer-bases-log2", type=int, default=28)
    ap.add_argument("--kmer-file", default=None,
                    help="--form kmer: insert the k-mers of this file (u64 count + u64 2-bit k-mers, the "
                         "reference's k-mer benchmark format) instead of synthetic DNA")
    ap.add_argument("--form", choices=("plain", "batched", "served", "kmer", "grid", "policies", "sharded", "gather",
                                       "lookup_paths"),
                    default="plain",
                    help="batched: the filter-set form over 4096 uneven filters; served: the multi-tenant "
                         "continuous-batching form; sharded: the hash-partitioned multi-GPU form (each its own "
                         "JSON line)")
    ap.add_argument("--routing", choices=("reference", "remixed"), default=None,
                    help="shard routing of CuckooFilterMultiGPU (default: reference for --form sharded, remixed for "
                         "the plain form on N GPUs)")
    ap.add_argument("--multi", choices=("auto", "sharded", "independent"), default="auto",
                    help="plain form on N GPUs: 'sharded' = one filter hash-partitioned over the GPUs "
                         "(CuckooFilterMultiGPU, NCCL all-to-all), 'independent' = one independent filter per GPU "
                         "with no collective; auto = sharded for N > 1, the single filter for N = 1")
    ap.add_argument("--shard-slots-log2", type=int, default=28, help="--form sharded: log2 slots per rank")
    ap.add_argument("--tenants", type=int, default=256)
    ap.add_argument("--loads", default="10,50,100,200", help="offered loads of the served form, Mkeys/s")
    ap.add_argument("--duration", type=float, default=0.5, help="seconds of arrivals per offered load")
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--filters", type=int, default=4096)
    ap.add_argument("--batched-seed", type=int, default=1)
    args = ap.parse_args()
    if args.warmup < 1:
        ap.error("--warmup must be >= 1")
    w = dict(WORKLOADS[args.workload])
    if args.bits:
        w["bits"], w["bs"] = args.bits, 8 if args.bits == 32 else 16
        w["desc"] += f" [bits per tag {w['bits']}, bucket size {w['bs']}]"
    if args.form == "batched":
        res = run_batched(args)
    elif args.form == "served":
        res = run_served(args)
    elif args.form == "kmer":
        res = run_kmer(args)
    elif args.form == "policies":
        res = run_policies(args)
    elif args.form == "grid":
        res = run_grid(args)
    elif args.form == "sharded":
        args.routing = args.routing or "reference"
        res = run_sharded(args)
    elif args.form == "gather":
        res = run_gather(args)
    elif args.form == "lookup_paths":
        res = run_lookup_paths(args, w)
    elif args.impl == "reference":
        res = run_reference(args, w)
    else:
        world = int(os.environ.get("WORLD_SIZE", "1"))
        sharded = args.multi == "sharded" or (args.multi == "auto" and world > 1)
        if sharded:
            args.routing = args.routing or "remixed"
            res = run_b200_sharded(args, w)
        else:
            res = run_b200(args, w)
            if res is not None and world == 1 and not args.no_forms:
                res["forms"] = run_forms_summary(args)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
