"""GPU parity of stratified negation: ``unreached(x, y) :- cand(x, y), !path(x, y).``

The reference evaluates this program only on GeneralCpu (the binary lowering
rejects the non-recursive derived predicate, subset.rs:56-63), so the oracle
is the nested-loop GeneralCpu restatement (small inputs) and the operator
pipeline anti_join(distinct(cand), path) pinned against it (larger inputs).
"""

import numpy as np
import pytest

import oracle
from conftest import pairs
from sparkalog_b200 import generators

pytestmark = pytest.mark.gpu

EDGE, PATH, CAND, UNREACHED = 0, 1, 2, 3


def program():
    from sparkalog_b200.datalog import BinarySccPlan, BinarySeedPlan, NegationClause
    from sparkalog_b200.recursion import transitive_closure_scc
    from sparkalog_b200.relational import RelationId as R

    tc = BinarySccPlan(transitive_closure_scc(R(PATH), R(EDGE)), [BinarySeedPlan(R(PATH), R(EDGE), (0, 1))])
    return [tc, NegationClause(R(UNREACHED), R(CAND), R(PATH))]


def run_device(src, dst, c0, c1):
    from sparkalog_b200.datalog import execute_stratified

    store, summaries = execute_stratified(4, program(), relations={EDGE: (src, dst), CAND: (c0, c1)})
    return store, summaries


def general_cpu(src, dst, c0, c1):
    facts = [(EDGE, (int(a), int(b))) for a, b in zip(src, dst)] + \
        [(CAND, (int(a), int(b))) for a, b in zip(c0, c1)]
    seed = oracle.Clause(PATH, [("b", 0), ("b", 1)], [oracle.Atom(EDGE, [("b", 0), ("b", 1)])])
    rec = oracle.Clause(PATH, [("b", 0), ("b", 2)], [oracle.Atom(PATH, [("b", 0), ("b", 1)], delta=True),
                                                      oracle.Atom(EDGE, [("b", 1), ("b", 2)])])
    neg = oracle.Clause(UNREACHED, [("b", 0), ("b", 1)], [oracle.Atom(CAND, [("b", 0), ("b", 1)])],
                        [oracle.Atom(PATH, [("b", 0), ("b", 1)])])
    strata = [[oracle.GeneralScc([PATH], True, [seed], [rec])], [oracle.GeneralScc([UNREACHED], False, [neg], [])]]
    return oracle.general_cpu(4, facts, strata)


@pytest.mark.parametrize("n,e,cands,seed", [(30, 25, 300, 1), (60, 90, 2000, 2), (12, 0, 50, 3)])
def test_negation_matches_general_cpu(cuda, n, e, cands, seed):
    src, dst = generators.er_edges(n, e, seed)
    c0, c1 = generators.uniform_pairs(n, cands, seed + 100)
    store, summaries = run_device(src, dst, c0, c1)
    full, want = general_cpu(src, dst, c0, c1)
    assert [tuple(p) for p in pairs(store.full(UNREACHED))] == sorted(full[UNREACHED])
    assert [tuple(p) for p in pairs(store.full(PATH))] == sorted(full[PATH])
    # Per-SCC summaries: (rows, iterations, new rows) as GeneralCpu reports them.
    assert [s.iterations for s in summaries] == [w[1] for w in want]
    assert [s.new_rows for s in summaries] == [w[2] for w in want]
    assert [[(r.value, k) for r, k in s.relations] for s in summaries] == [w[0] for w in want]


def test_negation_matches_operator_oracle_at_scale(cuda):
    src, dst = generators.er_edges(200_000, 175_000, 5)
    c0, c1 = generators.uniform_pairs(200_000, 1_000_000, 55)
    # Plant candidates that are reachable, so the anti-join removes some.
    (p0, p1), _, _ = oracle.transitive_closure(src, dst, threads=8)
    c0 = np.concatenate([c0, p0[::7]])
    c1 = np.concatenate([c1, p1[::7]])
    store, _ = run_device(src, dst, c0, c1)
    want = oracle.anti_join(oracle.distinct((c0, c1)), (p0, p1))
    got = store.full(UNREACHED)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_negation_edge_cases(cuda):
    from sparkalog_b200.datalog import NegationClause, execute_stratified
    from sparkalog_b200.relational import RelationId as R

    e = np.array([1, 2], dtype=np.uint32), np.array([2, 3], dtype=np.uint32)
    empty = np.zeros(0, dtype=np.uint32), np.zeros(0, dtype=np.uint32)
    # Empty candidates, and candidates all inside the negated relation.
    store, s = execute_stratified(4, [NegationClause(R(3), R(2), R(0))], relations={0: e, 2: empty})
    assert store.rows(3) == 0 and s[0].iterations == 1
    store, _ = execute_stratified(4, [NegationClause(R(3), R(2), R(0))], relations={0: e, 2: e})
    assert store.rows(3) == 0
    # Empty negated relation keeps every (deduplicated, sorted) candidate.
    c = np.array([5, 1, 5], dtype=np.uint32), np.array([6, 2, 6], dtype=np.uint32)
    store, _ = execute_stratified(4, [NegationClause(R(3), R(2), R(0))], relations={0: empty, 2: c})
    assert pairs(store.full(3)) == [[1, 2], [5, 6]]
