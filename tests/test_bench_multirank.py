"""The N>1 path of bench.py on CPU: two gloo ranks, each an independent filter
shard with its own key streams, aggregated as the whole job (keys of all
ranks over the slowest rank's time).  No GPU and no NCCL: the reductions run
over gloo exactly as they run over NCCL on GPUs."""
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
