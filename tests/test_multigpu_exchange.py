"""The hash-partitioned multi-GPU form (cuckoo-filter_b200/multigpu.py) on CPU
ranks: the exchange protocol over gloo, world sizes 2 and 3.

Each rank's device side (its filter shard and the grouping kernels) is
replaced by a host stand-in: the oracle as the shard, numpy grouping by the
library's host hash (``cf_hash64``) as the partition.  What runs unchanged is
the product's protocol: rounds agreed by all ranks, the all-to-all of counts,
keys and results, and the placement of results at their batch positions.
Checked against a global oracle: every key lands in the shard
hash64(key) % world; lookups and deletes answer in the caller's key order;
totals are sums over ranks; uneven and empty batches and multi-round batches
(different round counts per rank) work.
"""
from __future__ import annotations

import datetime
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CAP = 40_000


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class HostShardOps:
    """Host stand-in for DeviceShardOps (test infrastructure)."""

    device = torch.device("cpu")

    def __init__(self, orc, mg, capacity):
        self.mg = mg
        self.o = orc.OracleFilter(key_bytes=8, bits=16, bucket_size=16, policy=1, max_evictions=500,
                                  capacity=capacity, mode=orc.MODE_CONSERVING)
        self.stored = []

    def to_device(self, keys):
        return torch.from_numpy(np.ascontiguousarray(keys, dtype=np.uint64).view(np.int64))

    def partition(self, keys, ns, routing=0):
        a = keys.numpy().view(np.uint64)
        d = self.mg.shard_of(a, ns, routing=("reference", "remixed")[routing])
        order = np.argsort(d, kind="stable")
        counts = np.bincount(d, minlength=ns).astype(np.int64)
        return (torch.from_numpy(a[order].view(np.int64).copy()), torch.from_numpy(order.astype(np.int32)),
                torch.from_numpy(counts))

    def unpartition(self, grouped, pos):
        out = np.empty(grouped.numel(), np.uint8)
        out[pos.numpy()] = grouped.numpy()
        return torch.from_numpy(out)

    def insert(self, keys):
        a = keys.numpy().view(np.uint64)
        self.stored.append(a.copy())
        self.o.insert(a)

    def contains(self, keys):
        return torch.from_numpy(self.o.contains(keys.numpy().view(np.uint64)))

    def delete(self, keys):
        return torch.from_numpy(self.o.delete(keys.numpy().view(np.uint64))[1])

    def occupied(self):
        return self.o.occupied()

    def capacity(self):
        return self.o.nb * 16

    def size_in_bytes(self):
        return self.o.table.nbytes

    def clear(self):
        self.o.table[:] = 0

    def synchronize(self):
        pass


def _rank_main(rank, world, port, q, routing):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import oracle as orc
        from conftest import load_package

        cfb = load_package()
        import cuckoo_b200.multigpu as mg

        cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=16, bucketSize=16)
        ops = HostShardOps(orc, mg, mg.capacity_per_gpu(CAP, world))
        # small rounds, so that ranks with different batch sizes take several
        f = mg.CuckooFilterMultiGPU(cfg, CAP, ops=ops, max_keys_per_call=3000, routing=routing)
        # uneven batches; the last rank inserts nothing
        n = [9000, 4000, 0][rank] if world == 3 else [9000, 4000][rank]
        keys = orc.splitmix64(100 + rank, n)
        occ = f.insertMany(keys)
        mine = np.concatenate(ops.stored) if ops.stored else np.zeros(0, np.uint64)
        # lookups: this rank's keys, another rank's keys and negatives, shuffled
        other = orc.splitmix64(100 + (rank + 1) % world, 500)
        neg = orc.splitmix64(900 + rank, 700)
        qk = np.concatenate([keys[:1500], other, neg])
        np.random.default_rng(rank).shuffle(qk)
        got = f.containsMany(qk)
        # deletes of half of this rank's keys, results in the caller's order
        dels = keys[: n // 2]
        dout = np.zeros(len(dels), bool)
        occ2 = f.deleteMany(dels, dout)
        after = f.containsMany(keys[n // 2:])
        q.put((rank, occ, occ2, mine, qk, got, dout, after, f.totalCapacity(), f.sizeInBytes(),
               f.capacityPerGPU, ops.capacity(), f.loadFactor()))
        f.synchronizeAllGPUs()
    except BaseException:
        import traceback

        q.put((rank, "error", traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,routing", [(2, "reference"), (3, "reference"), (2, "remixed")])
def test_exchange_protocol_over_gloo(cfb, orc, world, routing):
    import cuckoo_b200.multigpu as mg

    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q, routing)) for r in range(world)]
    for p in procs:
        p.start()
    res = []
    for _ in range(world):
        r = q.get(timeout=240)
        assert r[1] != "error", f"rank {r[0]}:\n{r[2]}"
        res.append(r)
    res.sort(key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    sizes = [9000, 4000, 0][:world]
    all_keys = [orc.splitmix64(100 + r, sizes[r]) for r in range(world)]
    everything = np.concatenate(all_keys)
    owner = mg.shard_of(everything, world, routing=routing)
    for rank, occ, occ2, mine, qk, got, dout, after, tcap, tbytes, cpg, cap_r, lf in res:
        # the shard holds exactly the keys (of every rank) that hash to it
        assert np.array_equal(np.sort(mine), np.sort(everything[owner == rank])), rank
        # totals are sums over ranks, identical on every rank
        assert occ == len(everything) and occ2 == len(everything) - sum(s // 2 for s in sizes)
        assert tcap == sum(r[11] for r in res) and cpg == mg.capacity_per_gpu(CAP, world)
        assert lf == pytest.approx(occ2 / tcap)
        # lookups in the caller's order: every stored key (this rank's and
        # another rank's) is found at its own position; negatives are mostly not
        stored = np.isin(qk, everything)
        assert got[stored].all(), rank
        assert got[~stored].mean() < 0.01, rank
        assert dout.all() and after.all()
    assert len({r[8] for r in res}) == 1 and len({r[9] for r in res}) == 1


def test_capacity_per_gpu_matches_reference_rounding(cfb):
    import cuckoo_b200.multigpu as mg

    # static_cast<size_t>(SDIV(capacity, numGPUs) * 1.02)
    assert mg.capacity_per_gpu(1 << 20, 8) == int((1 << 17) * 1.02)
    assert mg.capacity_per_gpu(1000, 3) == int(334 * 1.02)
    assert mg.capacity_per_gpu(1, 4) == 1


def test_host_shard_of_is_hash_mod_n(cfb, orc):
    import cuckoo_b200.multigpu as mg

    keys = orc.splitmix64(5, 2000)
    want = np.array([orc.xxhash64(int(k), 8) % 7 for k in keys], np.int64)
    assert np.array_equal(mg.shard_of(keys, 7), want)
    k32 = keys.astype(np.uint32)
    want32 = np.array([orc.xxhash64(int(k), 4) % 5 for k in k32], np.int64)
    assert np.array_equal(mg.shard_of(k32, 5, key_bytes=4), want32)


def test_remixed_routing_keeps_buckets_independent(cfb, orc):
    """With the XOR policy and 8 shards, the reference's routing (hash % 8)
    leaves a shard's keys 1/8 of the buckets as primary buckets: filling one
    shard to 0.95 fails inserts and multiplies evictions.  The remixed routing
    fills it like an unsharded filter."""
    import cuckoo_b200.multigpu as mg

    cap = 1 << 18
    keys = orc.splitmix64(5, 8 * cap)
    res = {}
    for routing in ("reference", "remixed"):
        k0 = keys[mg.shard_of(keys, 8, routing=routing) == 0][: int(0.95 * cap)]
        o = orc.OracleFilter(key_bytes=8, bits=16, bucket_size=16, policy=1, max_evictions=500, capacity=cap,
                             mode=orc.MODE_CONSERVING)
        i1, _, _ = o.candidates(k0)
        res[routing] = (len(k0) - o.insert(k0), len(np.unique(i1)) / o.nb)
    assert res["reference"][1] <= 1 / 8 + 1e-9 and res["reference"][0] > 0
    assert res["remixed"][1] > 0.99 and res["remixed"][0] == 0
