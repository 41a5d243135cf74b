"""The N>1 paths of bench.py on CPU, two gloo ranks.

* independent shards: each rank an independent filter with its own key
  streams, aggregated as the whole job (keys of all ranks over the slowest
  rank's time);
* the hash-partitioned front end (the default for N > 1): the plain step's
  phases through CuckooFilterMultiGPU, each rank's shard a host stand-in.
No GPU and no NCCL: the collectives run over gloo exactly as they run over
NCCL on GPUs."""
from __future__ import annotations

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TINY = dict(capacity=1 << 14, bits=16, bs=16, policy="BFS", max_ev=500, fill=0.95,
            n_pos=1 << 11, n_neg=1 << 11, n_del=1 << 10, seed_fill=3, seed_neg=4, seed_sample=5)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        fill, query, dele, ncoll = bench.make_inputs(TINY, torch.device("cpu"), rank)
        # rank r's slowest time is 10 + r ms; each rank processed the same key count
        keys_per_step = fill.numel() + query.numel() + dele.numel()
        value, tmax = bench.aggregate(world, keys_per_step, 3, 10.0 + rank)
        q.put((rank, fill[:8].tolist(), int(fill.numel()), value, tmax, ncoll))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_aggregate():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(2))
    (r0, head0, n0, v0, t0, c0), (r1, head1, n1, v1, t1, c1) = res
    assert (r0, r1) == (0, 1)
    assert head0 != head1, "each rank draws its own key stream (seeds offset by rank)"
    assert n0 == n1 == int(0.95 * TINY["capacity"])
    # whole-job value: all ranks' keys over the slowest rank's time, identical on every rank
    keys = 2 * 3 * (n0 + TINY["n_pos"] + TINY["n_neg"] + TINY["n_del"])
    assert t0 == t1 == 11.0
    assert v0 == v1 == pytest.approx(keys / 11e-3 / 1e9)


def _sharded_rank_main(rank: int, world: int, port: int, q):
    """bench.sharded_step on one gloo rank: the plain workload's phases through
    CuckooFilterMultiGPU, each rank's shard a host stand-in (the oracle)."""
    import datetime
    import sys

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import oracle as orc
        from conftest import load_package
        from test_multigpu_exchange import HostShardOps

        cfb = load_package()
        import cuckoo_b200.multigpu as mg

        cap = bench.sharded_capacity(world, TINY["capacity"])
        cfg = cfb.CuckooConfig(T="uint64", bitsPerTag=16, bucketSize=16)
        ops = HostShardOps(orc, mg, mg.capacity_per_gpu(cap, world))
        f = mg.CuckooFilterMultiGPU(cfg, cap, ops=ops, routing="remixed", max_keys_per_call=1 << 31)
        fill, query, dele, _, is_pos = bench.make_inputs(TINY, torch.device("cpu"), rank, with_mask=True)
        marks = []
        q_out, d_out = bench.sharded_step(f, fill, query, dele, marks=marks.append)
        q.put((rank, ops.capacity(), int((is_pos & ~q_out).sum()), int(d_out.sum()), dele.numel(),
               f.totalOccupiedSlots(), fill.numel(), marks))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_run_the_sharded_plain_step():
    """The plain form on N ranks through the hash-partitioned front end: each
    rank's shard has the workload's capacity, every rank finds all of its own
    positives, removes all of its deletes, and the shards hold all the keys."""
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sharded_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(2))
    n_fill = 0
    for rank, shard_cap, missed, removed, n_del, total_occ, nf, marks in res:
        assert shard_cap == TINY["capacity"], "each rank's shard has the workload's capacity"
        assert missed == 0 and removed == n_del, (rank, missed, removed, n_del)
        assert marks == [0, 1, 2, 3]
        n_fill += nf
    assert res[0][5] == res[1][5] == n_fill - 2 * TINY["n_del"]
