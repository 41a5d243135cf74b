"""Serving form: many tenant filters, requests arriving over time, continuous
batching on one GPU.

The reference's server (CuckooFilterIPC.cuh:200-308) executes one request at
a time, synchronously.  This loop instead keeps every tenant's table resident
in a filter set (one set per tag width; ``CuckooFilterSet``) and, whenever the
device can take more work, forms a *wave* from every request that has arrived:
each tenant contributes the longest run of same-kind requests at the head of
its queue (lookups, inserts or deletes), so a tenant's operations are applied
in arrival order while different tenants' requests share one kernel launch per
kind.  Waves run back to back on one stream; the host builds wave k+1 (and
copies its keys in) while the GPU runs wave k.  A wave takes at most
``max_wave_keys`` keys (the staging slots): requests beyond that wait for the
next wave.  Tenants are admitted while their tables fit the HBM budget.

Results are exactly those of running each tenant's requests alone, in order,
through the single-filter API: a lookup or delete outcome depends only on the
multiset of (bucket pair, tag) entries of the tenant's table, which the same
sequence of operations evolves identically whatever else shares the wave.
"""
from __future__ import annotations

import collections
import dataclasses
import math
import time
from typing import Optional

import numpy as np

OP_LOOKUP, OP_INSERT, OP_DELETE = 0, 1, 2
OP_NAMES = {OP_LOOKUP: "lookup", OP_INSERT: "insert", OP_DELETE: "delete"}


@dataclasses.dataclass
class Tenant:
    tid: int
    capacity: int
    bits: int


@dataclasses.dataclass
class Request:
    rid: int
    tenant: int
    op: int
    keys: np.ndarray          # uint64 keys (host)
    arrival: float            # seconds from the start of the trace
    done: float = math.nan    # completion time (seconds from the start)
    result: Optional[np.ndarray] = None  # uint8 per key (lookups, deletes, inserts)


def splitmix64(seed: int, first: int, n: int) -> np.ndarray:
    """splitmix64(seed) outputs first .. first + n - 1 (uint64)."""
    G, M1, M2 = np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)
    with np.errstate(over="ignore"):
        z = (np.arange(first + 1, first + n + 1, dtype=np.uint64) * G) + np.uint64(seed)
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def make_tenants(n: int, seed: int, cap_lo: int = 16, cap_hi: int = 26) -> list[Tenant]:
    """Capacities log-uniform in 2^cap_lo..2^cap_hi slots; 8- or 16-bit tags."""
    rng = np.random.default_rng(seed)
    caps = np.exp2(rng.uniform(cap_lo, cap_hi, n)).astype(np.int64)
    bits = rng.choice([8, 16], n)
    return [Tenant(i, int(c), int(b)) for i, (c, b) in enumerate(zip(caps, bits))]


def make_trace(tenants: list[Tenant], rate_keys_per_s: float, duration_s: float, seed: int,
               median_keys: int = 16384, sigma: float = 1.0, lo: int = 1024, hi: int = 1 << 20,
               mix=(0.6, 0.3, 0.1)) -> list[Request]:
    """Poisson arrivals whose key rate is `rate_keys_per_s`; 60/30/10 lookup /
    insert / delete; sizes lognormal(median, sigma) clipped to [lo, hi]; keys
    from a per-tenant splitmix64 stream; deletes target keys the tenant
    inserted earlier in the trace, lookups are half inserted keys and half new."""
    rng = np.random.default_rng(seed)
    mean_size = float(np.clip(median_keys * math.exp(sigma * sigma / 2), lo, hi))
    req_rate = rate_keys_per_s / mean_size
    t, rid = 0.0, 0
    next_key = collections.defaultdict(int)       # next unused stream position per tenant
    inserted = collections.defaultdict(list)      # (first, n) ranges of inserted keys per tenant
    deleted_upto = collections.defaultdict(int)   # how many inserted keys were handed to deletes
    out = []
    while True:
        t += rng.exponential(1.0 / req_rate)
        if t >= duration_s:
            break
        ten = tenants[int(rng.integers(len(tenants)))]
        n = int(np.clip(rng.lognormal(math.log(median_keys), sigma), lo, hi))
        op = int(rng.choice(3, p=mix))
        seed_t = 0x5EED0000 + ten.tid
        if op == OP_INSERT or (op == OP_DELETE and sum(c for _, c in inserted[ten.tid]) - deleted_upto[ten.tid] < n):
            op = OP_INSERT
            n = min(n, max(0, int(0.5 * ten.capacity) - sum(c for _, c in inserted[ten.tid])))
            if n == 0:
                op = OP_LOOKUP
                n = int(np.clip(rng.lognormal(math.log(median_keys), sigma), lo, hi))
        if op == OP_INSERT:
            keys = splitmix64(seed_t, next_key[ten.tid], n)
            inserted[ten.tid].append((next_key[ten.tid], n))
            next_key[ten.tid] += n
        elif op == OP_DELETE:
            keys = _history(seed_t, inserted[ten.tid], deleted_upto[ten.tid], n)
            deleted_upto[ten.tid] += n
        else:
            have = sum(c for _, c in inserted[ten.tid])
            npos = min(n // 2, have)
            start = int(rng.integers(0, have - npos + 1)) if npos else 0
            pos = _history(seed_t, inserted[ten.tid], start, npos)
            neg = splitmix64(seed_t ^ 0xABCDEF, next_key[ten.tid] + 10_000_000, n - npos)
            keys = np.concatenate([pos, neg])
        out.append(Request(rid, ten.tid, op, keys.astype(np.uint64), t))
        rid += 1
    return out


def _history(seed: int, ranges: list, start: int, count: int) -> np.ndarray:
    """Keys start .. start + count - 1 of a tenant's insert history (the
    concatenation of its inserted stream ranges), generated on demand."""
    out, skip = [], start
    for first, c in ranges:
        if count == 0:
            break
        if skip >= c:
            skip -= c
            continue
        take = min(c - skip, count)
        out.append(splitmix64(seed, first + skip, take))
        count -= take
        skip = 0
    return np.concatenate(out) if out else np.zeros(0, np.uint64)


def latency_stats(reqs: list[Request]) -> dict:
    lat = np.array([r.done - r.arrival for r in reqs if not math.isnan(r.done)])
    keys = sum(len(r.keys) for r in reqs)
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs) if reqs else float("nan")
    return {"requests": len(reqs), "keys": keys, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
            "throughput_mkeys_s": keys / span / 1e6}


class Server:
    """Continuous-batching server over filter sets (see the module docstring)."""

    def __init__(self, cfb, tenants: list[Tenant], hbm_budget_bytes: int, max_wave_keys: int = 1 << 24,
                 device: int = 0):
        import torch

        self.cfb, self.torch = cfb, torch
        self.dev = torch.device("cuda", device)
        # admission: tenants in order while their tables fit the budget
        self.admitted, self.rejected = [], []
        used = 0
        for t in tenants:
            nb = cfb.CuckooFilter.calculateNumBuckets(t.capacity, 16)
            b = nb * 16 * t.bits // 8
            if used + b <= hbm_budget_bytes:
                self.admitted.append(t)
                used += b
            else:
                self.rejected.append(t)
        self.table_bytes = used
        self.sets, self.slot = {}, {}
        for bits in (8, 16):
            ts = [t for t in self.admitted if t.bits == bits]
            if not ts:
                continue
            cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=bits, bucketSize=16, evictionPolicy=cfb.EvictionPolicy.BFS)
            self.sets[bits] = cfb.CuckooFilterSet(cfg, [t.capacity for t in ts])
            for i, t in enumerate(ts):
                self.slot[t.tid] = (bits, i)
        self.max_wave_keys = max_wave_keys
        self.stream = torch.cuda.Stream(device=self.dev)
        # staging: device keys/outputs, pinned host keys/outputs, double-buffered
        self.d_keys = [torch.empty(max_wave_keys, dtype=torch.int64, device=self.dev) for _ in range(2)]
        self.d_out = [torch.empty(max_wave_keys, dtype=torch.uint8, device=self.dev) for _ in range(2)]
        self.h_keys = [torch.empty(max_wave_keys, dtype=torch.int64).pin_memory() for _ in range(2)]
        self.h_out = [torch.empty(max_wave_keys, dtype=torch.uint8).pin_memory() for _ in range(2)]
        self.waves = 0
        self.launches = 0

    def close(self):
        for s in self.sets.values():
            s.close()

    def warm_up(self) -> None:
        """Serve one throwaway key per (tag width, kind) and clear every table,
        so that the first measured requests do not pay one-time costs (kernel
        module loading, first use of the staging buffers).  The tables and the
        wave counters are left as after construction."""
        for bits in self.sets:
            tid = next(t for t, (b, _) in self.slot.items() if b == bits)
            for op in (OP_INSERT, OP_LOOKUP, OP_DELETE):
                r = Request(rid=-1, tenant=tid, op=op, keys=np.array([12345], np.uint64), arrival=0.0)
                ev, _ = self._launch_wave([r], 0)
                ev.synchronize()
        for st in self.sets.values():
            st.clear(stream=self.stream)
        self.torch.cuda.synchronize(self.dev)
        self.waves = 0
        self.launches = 0

    # -------------------------------------------------------------- waves
    def _form_wave(self, queues: dict) -> list[Request]:
        """Head run of same-kind requests of every tenant with pending work,
        within the staging limit."""
        wave, total = [], 0
        for tid in list(queues.keys()):
            q = queues[tid]
            if not q:
                continue
            op = q[0].op
            while q and q[0].op == op and total + len(q[0].keys) <= self.max_wave_keys:
                r = q.popleft()
                wave.append(r)
                total += len(r.keys)
            if total >= self.max_wave_keys:
                break
        return wave

    def _launch_wave(self, wave: list[Request], buf: int):
        """Stage keys, launch one set kernel per (tag width, kind), queue the
        result copy; returns the completion event and per-request spans."""
        torch = self.torch
        # layout: grouped by (bits, op) so each group is one contiguous item list
        groups = collections.defaultdict(list)
        for r in wave:
            bits, idx = self.slot[r.tenant]
            groups[(bits, r.op)].append((r, idx))
        hk = self.h_keys[buf]
        spans, pos = {}, 0
        layout = []
        for (bits, op), items in groups.items():
            g0 = pos
            offs, filt = [pos], []
            for r, idx in items:
                n = len(r.keys)
                hk[pos:pos + n].numpy()[:] = r.keys.view(np.int64)
                spans[r.rid] = (pos, n)
                pos += n
                offs.append(pos)
                filt.append(idx)
            layout.append((bits, op, g0, pos, offs, filt))
        s = self.stream
        with torch.cuda.stream(s):
            dk, do = self.d_keys[buf], self.d_out[buf]
            dk[:pos].copy_(hk[:pos], non_blocking=True)
            for bits, op, g0, g1, offs, filt in layout:
                d_offs = torch.tensor([o - g0 for o in offs], dtype=torch.int64).pin_memory().to(self.dev,
                                                                                              non_blocking=True)
                d_filt = torch.tensor(filt, dtype=torch.int32).pin_memory().to(self.dev, non_blocking=True)
                st = self.sets[bits]
                if op == OP_LOOKUP:
                    st.contains_async(dk[g0:g1], d_offs, d_filt, do[g0:g1], stream=s)
                elif op == OP_INSERT:
                    st.insert_async(dk[g0:g1], d_offs, d_filt, do[g0:g1], stream=s)
                else:
                    st.delete_async(dk[g0:g1], d_offs, d_filt, do[g0:g1], stream=s)
                self.launches += 1
            self.h_out[buf][:pos].copy_(do[:pos], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        self.waves += 1
        return ev, spans

    def run(self, trace: list[Request], t0: Optional[float] = None) -> list[Request]:
        """Serve a trace in real time (arrival times relative to t0)."""
        torch = self.torch
        reqs = [r for r in trace if r.tenant in self.slot]
        queues = collections.OrderedDict((t.tid, collections.deque()) for t in self.admitted)
        t0 = time.perf_counter() if t0 is None else t0
        i, inflight, buf = 0, collections.deque(), 0
        while i < len(reqs) or any(queues.values()) or inflight:
            now = time.perf_counter() - t0
            while i < len(reqs) and reqs[i].arrival <= now:
                queues[reqs[i].tenant].append(reqs[i])
                i += 1
            # retire finished waves
            while inflight and inflight[0][0].query():
                ev, spans, wave, b = inflight.popleft()
                tdone = time.perf_counter() - t0
                out = self.h_out[b]
                for r in wave:
                    p, n = spans[r.rid]
                    r.result = out[p:p + n].numpy().copy()
                    r.done = tdone
            # admit a new wave when a staging buffer is free (at most two in flight)
            if len(inflight) < 2 and any(queues.values()):
                wave = self._form_wave(queues)
                if wave:
                    ev, spans = self._launch_wave(wave, buf)
                    inflight.append((ev, spans, wave, buf))
                    buf ^= 1
                    continue
            if not inflight and i < len(reqs) and not any(queues.values()):
                time.sleep(max(0.0, min(reqs[i].arrival - now, 0.001)))
            elif inflight:
                time.sleep(0)  # yield; the GPU is busy
        torch.cuda.synchronize(self.dev)
        return reqs


def serve_plain(cfb, tenants: list[Tenant], trace: list[Request], device: int = 0) -> list[Request]:
    """Baseline: the plain single-filter API, one synchronous call per request
    in arrival order (a FIFO server like the reference's, CuckooFilterIPC.cuh:200-308)."""
    import torch

    dev = torch.device("cuda", device)
    filters = {}
    for t in tenants:
        cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=t.bits, bucketSize=16, evictionPolicy=cfb.EvictionPolicy.BFS)
        filters[t.tid] = cfb.CuckooFilter(cfg, t.capacity)
    maxn = max(len(r.keys) for r in trace)
    hk = torch.empty(maxn, dtype=torch.int64).pin_memory()
    ho = torch.empty(maxn, dtype=torch.uint8).pin_memory()
    dk = torch.empty(maxn, dtype=torch.int64, device=dev)
    do = torch.empty(maxn, dtype=torch.uint8, device=dev)
    s = torch.cuda.Stream(device=dev)
    reqs = [r for r in trace if r.tenant in filters]
    t0 = time.perf_counter()
    for r in reqs:
        while time.perf_counter() - t0 < r.arrival:
            pass
        n = len(r.keys)
        f = filters[r.tenant]
        hk[:n].numpy()[:] = r.keys.view(np.int64)
        with torch.cuda.stream(s):
            dk[:n].copy_(hk[:n], non_blocking=True)
        if r.op == OP_LOOKUP:
            f.containsMany(dk[:n], do[:n].view(torch.bool), stream=s)
        elif r.op == OP_INSERT:
            f.insertMany(dk[:n], stream=s, d_output=do[:n].view(torch.bool))
        else:
            f.deleteMany(dk[:n], do[:n].view(torch.bool), stream=s)
        with torch.cuda.stream(s):
            ho[:n].copy_(do[:n], non_blocking=True)
        s.synchronize()
        r.result = ho[:n].numpy().copy()
        r.done = time.perf_counter() - t0
    for f in filters.values():
        f.close()
    return reqs
