"""GPU parity of batched fixpoints: every instance of one batched run equals its
own serial run and the oracle, bit for bit, iteration counts included."""

import numpy as np
import pytest

import oracle
from conftest import pairs
from sparkalog_b200 import generators

pytestmark = pytest.mark.gpu


def instances_for(count, base_seed, n_max=2048):
    params = generators.batched_instances(count, base_seed, n_max=n_max)
    return [generators.er_edges(p.nodes, p.edges, p.seed) for p in params]


def test_batched_matches_oracle_and_serial(cuda):
    from sparkalog_b200.batched import BatchedTransitiveClosure

    inst = instances_for(60, 7, n_max=1024)
    # Edge cases: an empty instance, a single edge, a chain, a cycle.
    inst[3] = (np.zeros(0, dtype=np.uint32), np.zeros(0, dtype=np.uint32))
    inst[5] = (np.array([3], dtype=np.uint32), np.array([9], dtype=np.uint32))
    inst[8] = (np.arange(40, dtype=np.uint32), np.arange(1, 41, dtype=np.uint32))
    inst[9] = (np.arange(30, dtype=np.uint32), (np.arange(30, dtype=np.uint32) + 1) % 30)
    batch = BatchedTransitiveClosure(inst)
    results, summary = batch.run()
    serial = batch.run_serial()
    assert summary.iterations == max(r.iterations for r in results)
    for k, (s, d) in enumerate(inst):
        (w0, w1), it, new = oracle.transitive_closure(s, d)
        r = results[k]
        assert r.iterations == it, k
        assert r.new_rows == new, k
        assert np.array_equal(r.path[0], w0) and np.array_equal(r.path[1], w1), k
        assert serial[k].iterations == it and pairs(serial[k].path) == pairs(r.path), k


def test_batched_full_id_range(cuda):
    from sparkalog_b200.batched import BatchedTransitiveClosure

    # Node ids up to 2^14 - 1 and the largest instance tags.
    inst = [generators.er_edges(16384, 9000, s) for s in range(3)]
    batch = BatchedTransitiveClosure([(np.zeros(0, np.uint32), np.zeros(0, np.uint32))] * 4093 + inst)
    results, _ = batch.run()
    for k, (s, d) in enumerate(inst):
        (w0, w1), it, new = oracle.transitive_closure(s, d, threads=8)
        r = results[4093 + k]
        assert r.iterations == it and r.new_rows == new
        assert np.array_equal(r.path[0], w0) and np.array_equal(r.path[1], w1)
    assert all(r.iterations == 0 and len(r.path[0]) == 0 for r in results[:4093])
