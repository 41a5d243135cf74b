"""Serving form (cuckoo-filter_b200/serving.py).

CPU: the trace generator (Poisson arrivals, sizes clipped, deletes only of
keys the tenant inserted earlier) and wave formation (a tenant contributes only
the head run of same-kind requests, within the staging limit).

GPU: every request's result in the continuous-batching mix equals its result
when the tenant's requests run alone, in order, through the single-filter API;
tenants beyond the HBM budget are not admitted.
"""
from __future__ import annotations

import collections

import numpy as np
import pytest


@pytest.fixture(scope="module")
def srv(cfb):
    import cuckoo_b200.serving as s

    return s


def test_trace_properties(srv):
    tenants = srv.make_tenants(16, seed=3, cap_lo=12, cap_hi=16)
    tr = srv.make_trace(tenants, 20e6, 0.2, seed=4, median_keys=2048, lo=256, hi=8192)
    assert tr and all(a.arrival <= b.arrival for a, b in zip(tr, tr[1:]))
    assert all(256 <= len(r.keys) <= 8192 or r.op == srv.OP_INSERT for r in tr)
    ins = collections.defaultdict(set)
    for r in tr:
        if r.op == srv.OP_INSERT:
            ins[r.tenant].update(r.keys.tolist())
        elif r.op == srv.OP_DELETE:
            assert set(r.keys.tolist()) <= ins[r.tenant]
    kinds = collections.Counter(r.op for r in tr)
    assert kinds[srv.OP_LOOKUP] > kinds[srv.OP_INSERT] > kinds[srv.OP_DELETE] > 0


def test_wave_takes_head_runs_within_limit(srv):
    class Fake:
        max_wave_keys = 10

    R = srv.Request
    k = lambda n: np.zeros(n, np.uint64)  # noqa: E731
    queues = collections.OrderedDict()
    queues[0] = collections.deque([R(0, 0, 0, k(3), 0), R(1, 0, 0, k(2), 0), R(2, 0, 1, k(1), 0)])
    queues[1] = collections.deque([R(3, 1, 2, k(4), 0), R(4, 1, 2, k(4), 0)])
    wave = srv.Server._form_wave(Fake(), queues)
    # tenant 0: both lookups, not the insert behind them; tenant 1: one delete (limit 10 keys)
    assert [r.rid for r in wave] == [0, 1, 3]
    assert [r.rid for r in queues[0]] == [2] and [r.rid for r in queues[1]] == [4]


@pytest.mark.gpu
def test_mixed_results_equal_alone_results(cfb, srv):
    tenants = srv.make_tenants(24, seed=5, cap_lo=12, cap_hi=18)
    trace = srv.make_trace(tenants, 30e6, 0.25, seed=6, median_keys=4096, lo=512, hi=32768)
    server = srv.Server(cfb, tenants, hbm_budget_bytes=1 << 40, max_wave_keys=1 << 18)
    try:
        server.warm_up()  # leaves empty tables: the results below still equal the alone run's
        assert server.waves == 0 and int(sum(s.occupied().sum() for s in server.sets.values())) == 0
        served = server.run(trace)
    finally:
        server.close()
    assert server.waves > 1 and len(served) == len(trace)
    assert all(r.result is not None for r in served)
    # alone: each tenant's requests in order through the plain single-filter API
    import copy

    alone = srv.serve_plain(cfb, tenants, [copy.copy(r) for r in trace])
    by_rid = {r.rid: r for r in alone}
    for r in served:
        assert np.array_equal(r.result, by_rid[r.rid].result), (r.rid, r.tenant, srv.OP_NAMES[r.op])
    st = srv.latency_stats(served)
    assert st["p99_ms"] >= st["p50_ms"] > 0


@pytest.mark.gpu
def test_admission_by_hbm_budget(cfb, srv):
    tenants = srv.make_tenants(8, seed=7, cap_lo=16, cap_hi=20)
    sizes = [cfb.CuckooFilter.calculateNumBuckets(t.capacity, 16) * 2 * t.bits for t in tenants]
    budget = sum(sizes[:3])
    server = srv.Server(cfb, tenants, hbm_budget_bytes=budget, max_wave_keys=1 << 16)
    try:
        assert [t.tid for t in server.admitted] == [0, 1, 2]
        assert server.table_bytes <= budget and len(server.rejected) == 5
        trace = srv.make_trace(tenants, 5e6, 0.05, seed=8, median_keys=1024, lo=256, hi=4096)
        served = server.run(trace)
        assert {r.tenant for r in served} <= {0, 1, 2}
    finally:
        server.close()
