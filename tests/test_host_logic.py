"""CPU tests of host-side logic that needs no GPU: batching tags and splits,
workload generators, x-range partitioning."""

import numpy as np
import pytest

from sparkalog_b200 import generators, sharding


def test_batched_tagging_and_split():
    from sparkalog_b200.batched import BatchedTransitiveClosure

    inst = [(np.array([2, 0, 2], np.uint32), np.array([3, 1, 3], np.uint32)),
            (np.zeros(0, np.uint32), np.zeros(0, np.uint32)),
            (np.array([5], np.uint32), np.array([6], np.uint32))]
    b = BatchedTransitiveClosure(inst, id_bits=4)
    f, s = b.tagged_edges()
    assert f.tolist() == [0, 2, 32 + 5] and s.tolist() == [1, 3, 32 + 6]
    assert np.all(np.diff((f.astype(np.uint64) << np.uint64(32)) | s) > 0)
    seen = np.array([0, 0, 1], np.uint32)
    new = np.array([0, 0, 0], np.uint64)
    res = b.split(f, s, seen, new)
    assert [r.path[0].tolist() for r in res] == [[0, 2], [], [5]]
    assert [r.iterations for r in res] == [1, 0, 2]


def test_batched_rejects_out_of_range_ids():
    from sparkalog_b200.batched import BatchedTransitiveClosure

    with pytest.raises(ValueError):
        BatchedTransitiveClosure([(np.array([16], np.uint32), np.array([1], np.uint32))], id_bits=4)
    with pytest.raises(ValueError):
        BatchedTransitiveClosure([(np.zeros(0, np.uint32), np.zeros(0, np.uint32))] * 17, id_bits=28)


def test_batched_instance_parameters():
    params = generators.batched_instances(4096, 3)
    n = np.array([p.nodes for p in params])
    d = np.array([p.degree for p in params])
    assert n.min() >= 64 and n.max() <= 16384
    assert d.min() >= 0.5 and d.max() <= 1.2
    # log-uniform node counts: about half the instances below the geometric mean.
    assert 0.45 < np.mean(n < 1024) < 0.55
    assert generators.batched_instances(10, 3)[4] == params[4]


def test_served_requests_stream():
    reqs = generators.served_requests(2000, 500.0, 9)
    arrivals = np.array([r.arrival_s for r in reqs])
    assert np.all(np.diff(arrivals) > 0)
    assert abs(len(reqs) / arrivals[-1] - 500.0) < 50.0
    e = np.array([r.edges for r in reqs])
    assert e.min() >= 1000 and e.max() <= 4_000_000
    assert all(0.6 <= r.degree <= 0.95 for r in reqs)


def test_uniform_pairs_dedup_and_sorted():
    c0, c1 = generators.uniform_pairs(50, 5000, 1)
    packed = (c0.astype(np.uint64) << np.uint64(32)) | c1
    assert np.all(np.diff(packed) > 0)
    assert c0.max() < 50 and c1.max() < 50


def test_bench_partition_covers_every_row():
    import bench

    src, dst = generators.er_edges(1000, 3000, 4)
    parts = [bench.partition(src, dst, 1000, r, 3) for r in range(3)]
    assert sum(len(p[0]) for p in parts) == len(src)
    assert np.array_equal(np.concatenate([p[0] for p in parts]), src)
    # Ranges are balanced by seed rows and never split an x between ranks.
    bounds = sharding.balanced_bounds(src, 1000, 3)
    for r, (s, _) in enumerate(parts):
        if len(s):
            assert s.min() >= bounds[r] and s.max() < bounds[r + 1]
        assert abs(len(s) - len(src) / 3) <= 0.05 * len(src)


def test_bench_baseline_helpers_on_cpu():
    # The bench's CPU-side helpers (no GPU): the GeneralCpu baseline, converged
    # and extrapolated, the pipeline-byte formula and the profiled traffic.
    import bench
    import oracle

    src, dst = generators.er_edges(300, 280, 5)
    e0, _ = oracle.btree_pairs(src, dst)
    (_, _), it, new = oracle.transitive_closure(src, dst)
    g = bench.general_cpu_baseline((src, dst), len(e0) + new, new, time_cap_s=5.0)
    assert g["status"] == "run to the fixpoint" and g["cores"] == 1 and g["value"] > 0
    src, dst = generators.er_edges(2000, 8000, 1)
    g = bench.general_cpu_baseline((src, dst), 3_837_620, 3_829_620, time_cap_s=0.2)
    assert g["status"] == "not run (extrapolated)" and g["seconds"] > 0.2
    trace = [{"delta_rows": 10, "join_rows": 8, "unique_rows": 8, "new_rows": 7, "full_rows": 17}]
    assert bench.pipeline_bytes(trace) > 0
    traffic, source = bench.profiled_traffic("anti_join", 19.1e6)
    assert traffic is None or traffic > 0


def test_bench_reference_arm_line():
    # `bench.py --impl reference` needs no GPU: one JSON line with the keys the
    # bench contract names, on the small workload.
    import json
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    out = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--workload", "er_2000_8000",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] >= 1
    # The whole fixpoint is timed, and the config equals the GPU arm's.
    assert line["config"] == bench_config("er_2000_8000", 3_829_620, 13)


def bench_config(workload, derived, iterations):
    import bench

    nodes, edges, seed = bench.WORKLOADS[workload]
    return bench.workload_config(workload, nodes, edges, seed, derived, iterations)
