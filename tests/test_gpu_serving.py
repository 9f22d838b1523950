"""GPU tests of the continuous-batching server: each request's result (rows and
iteration count) is the same alone and in the mix."""

import numpy as np
import pytest

import oracle
from sparkalog_b200 import generators

pytestmark = pytest.mark.gpu


def make_requests(count, seed, e_max=20_000):
    params = generators.served_requests(count, 1000.0, seed, e_max=e_max)
    from sparkalog_b200.serving import ServeRequest

    return [ServeRequest(k, p.arrival_s, *generators.er_edges(p.nodes, p.edges, p.seed)) for k, p in enumerate(params)]


def _host(col):
    if hasattr(col, "is_cuda"):
        return col.cpu().numpy().view(np.uint32)
    return col


def check_against_alone(report, requests):
    by_id = {c.request_id: c for c in report.completions}
    assert sorted(by_id) == [r.request_id for r in requests]
    for r in requests:
        (w0, w1), it, new = oracle.transitive_closure(r.src, r.dst)
        c = by_id[r.request_id]
        assert c.iterations == it, r.request_id
        assert c.new_rows == new, r.request_id
        assert np.array_equal(_host(c.path[0]), w0) and np.array_equal(_host(c.path[1]), w1), r.request_id


def test_served_results_equal_alone(cuda):
    from sparkalog_b200.serving import FixpointServer, serve, serve_one_at_a_time

    reqs = make_requests(40, 3)
    server = FixpointServer()
    report = serve(reqs, server, realtime=False)
    server.close()
    check_against_alone(report, reqs)
    alone = serve_one_at_a_time(reqs, realtime=False)
    check_against_alone(alone, reqs)


def test_slot_reuse_after_purge(cuda):
    from sparkalog_b200.serving import FixpointServer, serve

    # 8 slots (29-bit ids) for 30 requests: slots are retired, purged and reused.
    reqs = make_requests(30, 11, e_max=5_000)
    server = FixpointServer(id_bits=29)
    report = serve(reqs, server, realtime=False)
    server.close()
    check_against_alone(report, reqs)


def test_budget_limits_concurrency(cuda):
    from sparkalog_b200.serving import FixpointServer, serve

    reqs = make_requests(12, 5, e_max=3_000)
    server = FixpointServer(budget_bytes=2e6)
    peak = []
    orig_step = server.step

    def step():
        peak.append(len(server.active))
        return orig_step()

    server.step = step
    report = serve(reqs, server, realtime=False)
    server.close()
    check_against_alone(report, reqs)
    assert max(peak) < len(reqs)


def test_realtime_stream_latencies(cuda):
    from sparkalog_b200.serving import FixpointServer, serve

    reqs = make_requests(20, 8, e_max=10_000)
    server = FixpointServer()
    report = serve(reqs, server, realtime=True)
    server.close()
    s = report.summary()
    assert s["requests"] == 20
    assert all(c.finished_s >= c.arrival_s for c in report.completions)
    assert s["p99_ms"] >= s["p50_ms"] > 0


def test_extract_segment_untagged_equals_masked_read(cuda):
    from sparkalog_b200.recursion import RelationStore

    rng = np.random.default_rng(17)
    shift = 20
    segs = rng.integers(0, 1 << (32 - shift), 5000).astype(np.uint32)
    first = (segs << np.uint32(shift)) | rng.integers(0, 1 << shift, 5000).astype(np.uint32)
    second = (segs << np.uint32(shift)) | rng.integers(0, 1 << shift, 5000).astype(np.uint32)
    store = RelationStore()
    empty = np.zeros(0, dtype=np.uint32)
    store.insert_static(0, (empty, empty))
    store.append(0, (first, second))  # sorted and deduplicated on the device
    mask = np.uint32((1 << shift) - 1)
    for seg in [int(segs[0]), int(segs[1]), (1 << (32 - shift)) - 1, 0]:
        t0, t1 = store.extract_segment(0, shift, seg)
        u0, u1 = store.extract_segment(0, shift, seg, untag=True)
        assert np.all((t0 >> np.uint32(shift)) == seg)
        assert np.array_equal(u0, t0 & mask) and np.array_equal(u1, t1 & mask)
    store.close()


def test_large_pageable_reads_equal_pinned_reads(cuda):
    """Reads above the staged-copy threshold (32 MiB per column) into pageable
    NumPy arrays equal a read into page-locked buffers."""
    import torch

    from sparkalog_b200.recursion import FULL, RelationStore

    rng = np.random.default_rng(23)
    n = 20_000_000
    first = rng.integers(0, 1 << 12, n).astype(np.uint32) << np.uint32(20)
    first |= rng.integers(0, 1 << 20, n).astype(np.uint32)
    second = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    store = RelationStore()
    empty = np.zeros(0, dtype=np.uint32)
    store.insert_static(0, (empty, empty))
    store.append(0, (first, second))
    rows = store.rows(0)
    p0 = torch.empty(rows, dtype=torch.int32, pin_memory=True)
    p1 = torch.empty(rows, dtype=torch.int32, pin_memory=True)
    store.read_into(0, FULL, p0, p1)
    f0, f1 = store.full(0)
    assert len(f0) == rows
    assert np.array_equal(f0, p0.numpy().view(np.uint32)) and np.array_equal(f1, p1.numpy().view(np.uint32))
    # Segment 0 under shift 31 (first < 2^31) holds about half of the rows
    # (10M, 40 MB a column): the staged path with the tag cleared.
    u0, u1 = store.extract_segment(0, 31, 0, untag=True)
    t0, t1 = store.extract_segment(0, 31, 0)
    assert len(u0) * 4 >= 32 << 20
    assert np.array_equal(u0, t0 & np.uint32(0x7FFFFFFF)) and np.array_equal(u1, t1 & np.uint32(0x7FFFFFFF))
    store.close()


@pytest.mark.parametrize("readout,rounds,batch_last", [("device", 1, False), ("host", 4, False), ("device", 8, False),
                                                      ("device", 4, True)])
def test_laned_server_results_equal_alone(cuda, readout, rounds, batch_last):
    # Size lanes on their own streams and threads (the last one batched, or
    # running its requests one at a time), several rounds per step (the
    # device-driven loop), results in device or host memory: every request's
    # rows and iteration count equal its run alone.
    from sparkalog_b200.serving import LanedServer, serve_laned, serve_one_at_a_time

    reqs = make_requests(40, 13, e_max=60_000)
    server = LanedServer(bounds=(6_000,), readout=readout, rounds_per_step=rounds, batch_last=batch_last)
    report = serve_laned(reqs, server, realtime=False)
    lanes = [len(lane.completions) for lane in server.lanes]
    server.close()
    check_against_alone(report, reqs)
    assert all(n > 0 for n in lanes)
    alone = serve_one_at_a_time(reqs, realtime=False, readout=readout)
    check_against_alone(alone, reqs)


def test_laned_server_realtime(cuda):
    from sparkalog_b200.serving import LanedServer, serve_laned

    reqs = make_requests(30, 21, e_max=40_000)
    server = LanedServer(bounds=(5_000,), readout="device", rounds_per_step=4)
    report = serve_laned(reqs, server, realtime=True)
    server.close()
    check_against_alone(report, reqs)
    s = report.summary()
    assert s["requests"] == 30 and s["p99_ms"] >= s["p50_ms"] > 0
