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


def check_against_alone(report, requests):
    by_id = {c.request_id: c for c in report.completions}
    assert sorted(by_id) == [r.request_id for r in requests]
    for r in requests:
        (w0, w1), it, new = oracle.transitive_closure(r.src, r.dst)
        c = by_id[r.request_id]
        assert c.iterations == it, r.request_id
        assert c.new_rows == new, r.request_id
        assert np.array_equal(c.path[0], w0) and np.array_equal(c.path[1], w1), r.request_id


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
