"""The hash-partitioned multi-GPU form on one B200.

* ``cf_shard_partition`` against numpy: per-shard counts, every key in the
  group of shard hash64(key) % N, positions a permutation that maps each
  grouped key back to its batch slot (1 to 256 shards, 4- and 8-byte keys,
  empty, single-key and multi-CTA batches);
* ``cf_shard_unpartition`` is the inverse placement;
* N shards emulated on one GPU with the product's grouping kernels (no
  collective, no rank waits on another): each shard filter holds exactly its
  keys, and lookups through partition -> shard -> unpartition equal the oracle
  on each shard's image, in the caller's order;
* ``CuckooFilterMultiGPU`` end to end over NCCL with one rank.
"""
from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from test_gpu_parity import dev, host_u8, image  # noqa: E402


def partition(mg, keys_d, ns, kb, routing=0):
    ops = mg.KeyGrouping(keys_d.device, kb)
    g, pos, counts = ops.partition(keys_d, ns, routing)
    torch.cuda.synchronize()
    return ops, g, pos, counts


@pytest.mark.parametrize("routing", [0, 1])
@pytest.mark.parametrize("kb", [8, 4])
@pytest.mark.parametrize("ns", [1, 2, 3, 8, 256])
@pytest.mark.parametrize("n", [0, 1, 1000, 3_000_017])
def test_partition_groups_by_shard(cfb, orc, kb, ns, n, routing):
    import cuckoo_b200.multigpu as mg

    keys = orc.splitmix64(7 + ns, n)
    if kb == 4:
        keys = keys.astype(np.uint32)
    d = dev(keys)
    ops, g, pos, counts = partition(mg, d, ns, kb, routing)
    want = mg.shard_of(keys, ns, key_bytes=kb, routing=("reference", "remixed")[routing])
    c = counts.cpu().numpy()
    assert np.array_equal(c, np.bincount(want, minlength=ns)), "per-shard counts"
    gk = g.cpu().numpy().view(keys.dtype)
    p = pos.cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(p), np.arange(n)), "positions are a permutation"
    assert np.array_equal(gk, keys[p]), "grouped key i is batch key pos[i]"
    starts = np.concatenate([[0], np.cumsum(c)])
    for s in range(ns):
        assert (want[p[starts[s]:starts[s + 1]]] == s).all(), s
    r = torch.randint(0, 256, (n,), dtype=torch.uint8, device="cuda")
    back = ops.unpartition(r, pos)
    b = host_u8(back)
    want_b = np.empty(n, np.uint8)
    want_b[p] = host_u8(r)
    assert np.array_equal(b, want_b)


@pytest.mark.parametrize("ns,routing", [(2, 0), (4, 0), (7, 0), (4, 1), (8, 1)])
def test_emulated_shards_on_one_gpu(cfb, orc, ns, routing):
    import cuckoo_b200.multigpu as mg

    cap = 1 << 20
    cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=16, bucketSize=16)
    cpg = mg.capacity_per_gpu(cap, ns)
    shards = [cfb.CuckooFilter(cfg, cpg) for _ in range(ns)]
    keys = orc.splitmix64(40 + ns, int(0.9 * cap))
    rname = ("reference", "remixed")[routing]
    ops, g, pos, counts = partition(mg, dev(keys), ns, 8, routing)
    c = counts.cpu().tolist()
    starts = np.concatenate([[0], np.cumsum(c)]).astype(np.int64)
    ok = torch.empty(len(keys), dtype=torch.uint8, device="cuda")
    for s in range(ns):
        part = g[starts[s]:starts[s + 1]]
        shards[s].insertMany(part, d_output=ok[starts[s]:starts[s + 1]])
        st = shards[s].stats()
        assert shards[s].occupiedSlots() + st["failed"] == c[s] and st["lost"] == 0
        if routing == 1:
            assert st["failed"] == 0
    stored_g = host_u8(ok).astype(bool)
    gk = g.cpu().numpy().view(np.uint64)
    owner = mg.shard_of(keys, ns, routing=rname)
    q = np.concatenate([keys[::5], orc.splitmix64(99, 300_000)])
    qo = mg.shard_of(q, ns, routing=rname)
    ops2, gq, posq, cq = partition(mg, dev(q), ns, 8, routing)  # ops2 keeps q's run starts
    cqs = np.concatenate([[0], np.cumsum(cq.cpu().numpy())]).astype(np.int64)
    res = torch.empty(len(q), dtype=torch.uint8, device="cuda")
    for s in range(ns):
        if cqs[s + 1] > cqs[s]:
            shards[s].containsMany(gq[cqs[s]:cqs[s + 1]], res[cqs[s]:cqs[s + 1]])
    got = host_u8(ops2.unpartition(res, posq))
    want = np.empty(len(q), np.uint8)
    for s in range(ns):
        o = orc.OracleFilter(key_bytes=8, bits=16, bucket_size=16, policy=1, max_evictions=500, capacity=cpg,
                             mode=orc.MODE_CONSERVING)
        o.table[:] = image(shards[s])
        sel = qo == s
        want[sel] = o.contains(q[sel])
        # every key the shard stored is found there
        sel_g = np.zeros(len(gk), bool)
        sel_g[starts[s]:starts[s + 1]] = True
        assert o.contains(gk[sel_g & stored_g]).all()
        assert (owner[np.isin(keys, gk[sel_g])] == s).all()
    assert np.array_equal(got, want)
    for f in shards:
        f.close()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_front_end_over_nccl_one_rank(cfb, orc):
    import torch.distributed as dist

    import cuckoo_b200.multigpu as mg

    if dist.is_initialized():
        pytest.skip("a process group is already initialized")
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", 0))
    try:
        cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=16, bucketSize=16)
        f = mg.CuckooFilterMultiGPU(cfg, 1 << 20, max_keys_per_call=300_000)
        keys = orc.splitmix64(3, 900_000)
        occ = f.insertMany(keys)  # host keys, three rounds
        assert occ == len(keys) == f.totalOccupiedSlots()
        q = np.concatenate([keys[:200_000], orc.splitmix64(4, 200_000)])
        got = f.containsMany(q)
        o = orc.OracleFilter(key_bytes=8, bits=16, bucket_size=16, policy=1, max_evictions=500,
                             capacity=f.capacityPerGPU, mode=orc.MODE_CONSERVING)
        o.table[:] = image(f.ops.filter)
        assert got.dtype == bool and np.array_equal(got.astype(np.uint8), o.contains(q))
        dgot = f.containsMany(dev(q))  # device keys give a device result
        assert dgot.is_cuda and np.array_equal(host_u8(dgot), o.contains(q))
        out = np.zeros(100_000, bool)
        occ2 = f.deleteMany(keys[:100_000], out)
        assert out.all() and occ2 == len(keys) - 100_000
        assert f.totalCapacity() == f.ops.filter.capacity() and f.loadFactor() == pytest.approx(occ2 / f.totalCapacity())
        f.synchronizeAllGPUs()
        f.clear()
        assert f.totalOccupiedSlots() == 0
    finally:
        dist.destroy_process_group()
