"""The whole semi-naive loop on the reference's own CUDA operators agrees with
the device-resident executor, round by round.

The reference's column_ops.cu (crates/sparkalog-execution/native/column_ops.cu),
built unmodified for sm_100a into the oracle's ``_ref`` folder, exports the
same operator ABI as this library. The Tier A wrappers in
``sparkalog_b200.execution`` are pointed at it, and the loop below is
RecursiveExecutor::run's GPU path for transitive closure
(crates/sparkalog-recursion/src/generic.rs:197-397 for evaluate, combine and
apply, :472-516 for the loop): join DELTA with the edge index, distinct,
anti-join against FULL, union into FULL, DELTA = NEWT, one iteration per
executed round. Every kernel of that loop is the reference's; its per-round
cardinalities and final FULL must equal the executor's trace and FULL.
"""

import types

import numpy as np
import pytest
import torch

import oracle
from sparkalog_b200 import generators

pytestmark = pytest.mark.gpu


@pytest.fixture
def reference_operators(cuda, monkeypatch):
    ref = oracle.reference_cuda()
    if ref is None:
        pytest.skip("reference CUDA library not built (oracle/_ref)")
    from sparkalog_b200 import _native, execution

    _native.declare_operator_abi(ref)
    monkeypatch.setattr(execution, "_native", types.SimpleNamespace(load=lambda: ref))
    return execution


def reference_fixpoint(E, e0, e1):
    """RecursiveExecutor::run for path(x, z) :- path(x, y), edge(y, z) over the
    operator ABI; FULL and DELTA start as the sorted distinct edges."""
    from sparkalog_b200.relational import BinaryDistinct, SortedBinaryAntiJoin, SortedBinaryUnion, path_join

    stream = E.CudaStream()
    edge = E.Relation.from_host(e0, e1)
    index = E.U32RangeIndex(e0)  # U32RangeIndex::build_slice over edge column 0
    full = E.Relation.from_host(e0, e1)
    delta = E.Relation.from_host(e0, e1)
    wj, wd, wa = E.JoinWorkspace(), E.DistinctWorkspace(), E.AntiJoinWorkspace()
    # Uploads and clones run on torch's stream, the operators on their own.
    torch.cuda.synchronize()
    trace = []
    while len(delta):
        E.join_cuda(delta, edge, index, path_join(), wj, stream)
        E.distinct_cuda(wj.output, BinaryDistinct(), wd, stream)
        E.anti_join_cuda(wd.output, full, SortedBinaryAntiJoin(), wa, stream)
        newt = E.Relation(wa.output.columns[0].clone(), wa.output.columns[1].clone(), len(wa.output))
        wu = E.UnionWorkspace()
        torch.cuda.synchronize()
        E.union_cuda(full, newt, SortedBinaryUnion(), wu, stream)
        trace.append((len(delta), len(wj.output), len(wd.output), len(newt), len(wu.output)))
        full, delta = wu.output, newt
    return full.to_host(), trace


@pytest.mark.parametrize("nodes,edges,seed", [(2_000, 8_000, 1), (262_144, 229_376, 9)])
def test_reference_operator_loop_equals_executor(reference_operators, nodes, edges, seed):
    from sparkalog_b200 import recursion as R
    from sparkalog_b200.relational import RelationId

    src, dst = generators.er_edges(nodes, edges, seed)
    e0, e1 = oracle.btree_pairs(src, dst)
    (f0, f1), ref_trace = reference_fixpoint(reference_operators, e0, e1)

    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    ex = R.RecursiveExecutor.compile(R.transitive_closure_scc(RelationId(1), RelationId(0)), store)
    summary = ex.run(store, 10_000)
    got = [(r["delta_rows"], r["join_rows"], r["unique_rows"], r["new_rows"], r["full_rows"]) for r in ex.trace()]
    g0, g1 = store.full(1)
    ex.close()
    store.close()

    assert summary.iterations == len(ref_trace)
    assert got == ref_trace
    assert np.array_equal(g0, f0) and np.array_equal(g1, f1)
