"""GPU parity of general non-recursive clauses against GeneralCpu.

The reference evaluates non-recursive and negated clauses only on GeneralCpu
(crates/sparkalog-datalog/src/general.rs:478-551; the binary lowering rejects
them, subset.rs:56-63). Here each program is run by execute_stratified on the
device and by the oracle's nested-loop GeneralCpu restatement, and every
relation and per-SCC summary must be equal: constants in atoms and heads
(the reference's equality filter), repeated bindings, joins of two atoms,
negation in either binding order, several clauses for one target, a target
that also has facts, and clauses over a recursive relation's result.
"""

import numpy as np
import pytest

import oracle
from conftest import pairs
from sparkalog_b200 import generators

pytestmark = pytest.mark.gpu

A, B, C, EDGE, PATH, H1, H2, H3 = range(8)


def b(i):
    return ("b", i)


def v(x):
    return ("v", x)


def run_both(rels, clauses_by_target, facts=(), recursive=False):
    """clauses_by_target: [(target, [(head, positive, negative)])] in stratum order."""
    from sparkalog_b200.datalog import (BinarySccPlan, BinarySeedPlan, GeneralClause, NonRecursiveScc,
                                        PlannedAtom, execute_stratified)
    from sparkalog_b200.recursion import transitive_closure_scc
    from sparkalog_b200.relational import RelationId as R

    strata, ostrata = [], []
    if recursive:
        strata.append(BinarySccPlan(transitive_closure_scc(R(PATH), R(EDGE)), [BinarySeedPlan(R(PATH), R(EDGE), (0, 1))]))
        seed = oracle.Clause(PATH, [b(0), b(1)], [oracle.Atom(EDGE, [b(0), b(1)])])
        rec = oracle.Clause(PATH, [b(0), b(2)], [oracle.Atom(PATH, [b(0), b(1)], delta=True),
                                                  oracle.Atom(EDGE, [b(1), b(2)])])
        ostrata.append([oracle.GeneralScc([PATH], True, [seed], [rec])])
    for target, clauses in clauses_by_target:
        gcs, ocs = [], []
        for head, positive, negative in clauses:
            gcs.append(GeneralClause(R(target), tuple(head), tuple(PlannedAtom(R(r), tuple(t)) for r, t in positive),
                                     tuple(PlannedAtom(R(r), tuple(t)) for r, t in negative)))
            ocs.append(oracle.Clause(target, list(head), [oracle.Atom(r, list(t)) for r, t in positive],
                                     [oracle.Atom(r, list(t)) for r, t in negative]))
        strata.append(NonRecursiveScc(R(target), tuple(gcs)))
        ostrata.append([oracle.GeneralScc([target], False, ocs, [])])
    store, summaries = execute_stratified(8, strata, facts=[(R(r), t) for r, t in facts], relations=rels)
    ofacts = [(r, (int(x), int(y))) for r, (c0, c1) in rels.items() for x, y in zip(c0, c1)] + list(facts)
    full, want = oracle.general_cpu(8, ofacts, ostrata)
    for target, _ in clauses_by_target:
        assert [tuple(p) for p in pairs(store.full(target))] == sorted(full[target]), target
    assert [s.iterations for s in summaries] == [w[1] for w in want]
    assert [s.new_rows for s in summaries] == [w[2] for w in want]
    assert [[(r.value, k) for r, k in s.relations] for s in summaries] == [w[0] for w in want]
    store.close()


def rels(seed, n=400, hi=40):
    rng = np.random.default_rng(seed)
    out = {}
    for r in (A, B, C):
        x = rng.integers(0, hi, size=(n, 2)).astype(np.uint32)
        out[r] = (x[:, 0], x[:, 1])
    return out


@pytest.mark.parametrize("seed", [1, 2])
def test_constants_repeats_and_head_constants(cuda, seed):
    run_both(rels(seed), [
        (H1, [([b(0), v(7)], [(A, [b(0), b(1)])], [])]),          # h(x, 7) :- a(x, y)
        (H2, [([b(0), b(0)], [(A, [b(0), b(0)])], [])]),          # h(x, x) :- a(x, x)
        (H3, [([b(1), b(0)], [(B, [v(3), b(0)]), (C, [b(1), b(0)])], [])]),  # h(y, x) :- b(3, x), c(y, x)
    ])


@pytest.mark.parametrize("seed", [3, 4])
def test_join_with_negation_either_order(cuda, seed):
    run_both(rels(seed), [
        (H1, [([b(0), b(2)], [(A, [b(0), b(1)]), (B, [b(1), b(2)])], [(C, [b(0), b(2)])])]),
        (H2, [([b(1), b(0)], [(A, [b(0), b(1)])], [(B, [b(0), b(1)]), (C, [b(1), b(0)])])]),
    ])


def test_several_clauses_and_facts(cuda):
    r = rels(5)
    run_both(r, [
        (H1, [([b(0), b(1)], [(A, [b(0), b(1)])], [(B, [b(0), b(1)])]),
              ([b(1), b(0)], [(C, [b(0), b(1)])], []),
              ([v(1), b(0)], [(A, [b(0), v(2)]), (B, [b(0), b(3)])], [])]),
        (H2, [([b(0), b(1)], [(H1, [b(0), b(1)])], [(A, [b(0), b(1)])])]),
    ], facts=[(H1, (100, 200)), (H1, (3, 4))])


def test_clauses_over_a_recursive_result(cuda):
    src, dst = generators.er_edges(60, 70, 9)
    r = rels(6, n=300, hi=60)
    r[EDGE] = (src, dst)
    run_both(r, [
        (H1, [([b(0), b(1)], [(A, [b(0), b(1)])], [(PATH, [b(0), b(1)])])]),
        (H2, [([b(0), b(2)], [(PATH, [b(0), b(1)]), (B, [b(1), b(2)])], [(PATH, [b(0), b(2)])])]),
    ], recursive=True)


def test_unsupported_shapes_raise(cuda):
    from sparkalog_b200.datalog import GeneralClause, NonRecursiveScc, PlannedAtom, UnsupportedClause, \
        execute_stratified
    from sparkalog_b200.relational import RelationId as R

    bad = [GeneralClause(R(H1), (b(0), b(3)), (PlannedAtom(R(A), (b(0), b(1))), PlannedAtom(R(B), (b(2), b(3))))),
           GeneralClause(R(H1), (b(0), b(1)), (PlannedAtom(R(A), (b(0), b(1))),), (PlannedAtom(R(B), (b(0), v(1))),))]
    for clause in bad:
        with pytest.raises(UnsupportedClause):
            execute_stratified(8, [NonRecursiveScc(R(H1), (clause,))], relations=rels(7))
