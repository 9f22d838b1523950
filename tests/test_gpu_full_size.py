"""Bit-exact parity at the benchmark's full sizes (configs 2, 3 and 5).

The oracle's outputs at these sizes are gigabytes and take it minutes, so
they are pinned by digests: ``tests/golden/full_size.py`` runs the oracle on
each workload and commits, per relation, the SHA-256 of its sorted columns
together with the iteration and derived-row counts
(``tests/golden/full_size_digests.json``). Here the device runs the same
seeded workload through the public API, and the digest of every output must
equal the oracle's: equal digests mean equal rows in equal order.

* 16,777,216-node / 14,680,064-edge ER transitive closure (86 rounds), under
  the built-in tuning and under a second tuning (fine directories, small
  search groups, another level ratio), which must not change a bit;
* the stratified-negation workload (8,388,608 / 7,340,032 ER graph, then
  5.0e7 raw candidate pairs minus path);
* the 4,096-instance batched run: every instance's rows, iteration count and
  derived-row count.
"""

import json
import sys

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

sys.path.insert(0, str(GOLDEN))
import full_size  # noqa: E402


def digests() -> dict:
    return json.loads(full_size.DIGESTS.read_text())


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _tc(torch, src, dst, tuning=None):
    from sparkalog_b200.recursion import RecursiveExecutor, RelationStore, transitive_closure_scc
    from sparkalog_b200.relational import RelationId

    e0, e1 = _dev(torch, src), _dev(torch, dst)
    store = RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    ex = RecursiveExecutor.compile(transitive_closure_scc(RelationId(1), RelationId(0)), store)
    if tuning:
        ex.set_tuning(tuning)
    summary = ex.run(store)
    ex.close()
    return store, summary


@pytest.mark.parametrize("tuning", [None, {"dir_rows_log2": 2, "group_lanes": 4, "group_candidates": 1 << 20,
                                           "level_ratio": 6, "fused_rows_cap": 384, "levels": 4}])
def test_er_16m_transitive_closure_matches_oracle_digest(cuda, tuning):
    from sparkalog_b200 import generators

    want = digests()["er_16m"]
    src, dst = generators.er_edges(want["nodes"], want["edges"], want["seed"])
    store, summary = _tc(cuda, src, dst, tuning)
    try:
        assert summary.iterations == want["iterations"] == 86
        assert summary.total_new_rows == want["new_rows"]
        assert store.rows(1) == want["rows"]
        f0, f1 = store.full(1)
        assert full_size.pair_digest(f0, f1) == want["digest"]
    finally:
        store.close()


def test_negation_8m_matches_oracle_digest(cuda):
    from sparkalog_b200 import generators
    from sparkalog_b200.datalog import BinarySccPlan, BinarySeedPlan, NegationClause, execute_stratified
    from sparkalog_b200.recursion import transitive_closure_scc
    from sparkalog_b200.relational import RelationId as R

    want = digests()["negation_8m"]
    src, dst = generators.er_edges(want["nodes"], want["edges"], want["seed"])
    c0, c1 = full_size.negation_candidates(want["nodes"], want["cand_pairs"], want["cand_seed"])
    program = [BinarySccPlan(transitive_closure_scc(R(1), R(0)), [BinarySeedPlan(R(1), R(0), (0, 1))]),
               NegationClause(R(3), R(2), R(1))]
    store, summaries = execute_stratified(4, program, relations={0: (src, dst), 2: (c0, c1)})
    try:
        assert summaries[0].iterations == want["iterations"]
        assert summaries[0].new_rows == want["new_rows"]
        assert store.rows(1) == want["path_rows"]
        assert full_size.pair_digest(*store.full(1)) == want["path_digest"]
        assert store.rows(3) == want["unreached_rows"]
        assert full_size.pair_digest(*store.full(3)) == want["unreached_digest"]
    finally:
        store.close()


def test_batched_4096_every_instance_matches_oracle_digest(cuda):
    from sparkalog_b200.batched import BatchedTransitiveClosure

    want = digests()["batched_4096"]
    inst = full_size.batched_edges()
    assert len(inst) == want["count"] == 4096
    results, summary = BatchedTransitiveClosure(inst).run()
    assert summary.iterations == max(r[0] for r in want["instances"])
    assert sum(r.new_rows for r in results) == want["new_rows"]
    bad = []
    for k, (r, (it, new, rows, digest)) in enumerate(zip(results, want["instances"])):
        if (r.iterations, r.new_rows, len(r.path[0])) != (it, new, rows) or \
                full_size.pair_digest(*r.path) != digest:
            bad.append(k)
    assert not bad, f"{len(bad)} instances differ, first {bad[:10]}"
