"""GPU parity of the device-resident fixpoint (Tier B) against the oracle.

Mirrors crates/sparkalog-recursion/src/generic.rs:716-946 and
crates/sparkalog-datalog/src/subset.rs:475-497: FULL of every SCC relation
and the per-SCC iteration count must match bit for bit.
"""

import numpy as np
import pytest

import oracle
from conftest import cols, pairs
from sparkalog_b200 import generators

pytestmark = pytest.mark.gpu


def rec():
    from sparkalog_b200 import recursion

    return recursion


def plan_for(case):
    from sparkalog_b200.relational import RecursiveRulePlan, RecursiveSccPlan, RelationId, path_join

    rules = [RecursiveRulePlan(RelationId(r["target"]), RelationId(r["delta_input"]), RelationId(r["right_input"]),
                               path_join()) for r in case["rules"]]
    return RecursiveSccPlan([RelationId(r) for r in case["scc"]], rules)


def test_fixpoint_known_answers(cuda, known_answers):
    R = rec()
    for case in known_answers["fixpoint"]:
        store = R.RelationStore()
        for rid, rows in case["relations"].items():
            store.insert_static(int(rid), cols(rows))
        for rid, fd in case["recursive"].items():
            store.insert_recursive(int(rid), cols(fd["full"]), cols(fd["delta"]))
        ex = R.RecursiveExecutor.compile(plan_for(case), store)
        summary = ex.run(store, 16)
        if "iterations" in case:
            assert summary.iterations == case["iterations"], case["source"]
        if "total_new_rows" in case:
            assert summary.total_new_rows == case["total_new_rows"], case["source"]
        for rid, rows in case["full"].items():
            assert pairs(store.full(int(rid))) == rows, case["source"]
            assert store.rows(int(rid), R.DELTA) == 0
        assert [(r.value, n) for r, n in summary.relation_rows] == [
            (int(rid), len(case["full"][str(rid)])) for rid in case["scc"]]


def test_incompatible_plans_rejected(cuda):
    # generic.rs:917-946
    R = rec()
    from sparkalog_b200.relational import SortedBinaryUnion

    store = R.RelationStore()
    store.insert_static(0, cols([[1, 2]]))
    store.insert_recursive(1, cols([[1, 2]]), cols([[1, 2]]))
    plan = plan_for({"scc": [1], "rules": [{"target": 1, "delta_input": 1, "right_input": 0}] * 2})
    plan.rules[1].union = SortedBinaryUnion(left=(0, 1), right=(1, 0))
    with pytest.raises(R.GenericExecutionError) as err:
        R.RecursiveExecutor.compile(plan, store)
    assert err.value.kind == "IncompatibleTargetPlans"


def test_iteration_limit_and_store_errors(cuda):
    R = rec()
    store = R.RelationStore()
    e = cols([[i, i + 1] for i in range(10)])
    store.insert_static(0, e)
    store.insert_recursive(1, e, e)
    with pytest.raises(R.GenericExecutionError) as err:
        store.insert_static(0, e)
    assert err.value.kind == "Duplicate"
    with pytest.raises(R.GenericExecutionError) as err:
        store.rows(7)
    assert err.value.kind == "Missing"
    ex = R.RecursiveExecutor.compile(R.transitive_closure_scc(*map(_rid, (1, 0))), store)
    with pytest.raises(R.GenericExecutionError) as err:
        ex.run(store, 3)
    assert err.value.kind == "IterationLimit"


def _rid(v):
    from sparkalog_b200.relational import RelationId

    return RelationId(v)


@pytest.mark.parametrize("n", [2, 3, 17, 512])
def test_chain_closure(cuda, n):
    # tc-fixpoint.rs:118-154
    R = rec()
    src = np.arange(n - 1, dtype=np.uint32)
    store = R.RelationStore()
    store.insert_static(0, (src, src + 1))
    store.insert_recursive(1, (src, src + 1), (src, src + 1))
    summary = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store).run(store, 1024)
    assert store.rows(1) == n * (n - 1) // 2
    assert store.rows(1, R.DELTA) == 0
    assert summary.iterations == n - 1


def run_tc_gpu(src, dst, max_iterations=10_000):
    R = rec()
    e0, e1 = oracle.btree_pairs(src, dst)
    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    summary = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store).run(store,
                                                                                                 max_iterations)
    return store.full(1), summary


@pytest.mark.parametrize("n,e,seed", [(40, 60, 9), (2000, 8000, 1), (5000, 4500, 2), (300_000, 262_500, 6),
                                      (1_000, 1_000, 7)])
def test_tc_matches_oracle(cuda, n, e, seed):
    src, dst = generators.er_edges(n, e, seed)
    (p0, p1), summary = run_tc_gpu(src, dst)
    (w0, w1), it, new = oracle.transitive_closure(src, dst, threads=8)
    assert summary.iterations == it
    assert summary.total_new_rows == new
    assert np.array_equal(p0, w0) and np.array_equal(p1, w1)


def test_tc_seed_with_duplicates_and_unsorted_delta(cuda):
    # FULL may hold duplicates (the first union removes them) and DELTA's
    # order does not matter: distinct sorts the join output.
    R = rec()
    e0, e1 = cols([[1, 2], [2, 3], [3, 4], [4, 5], [5, 6]])
    full = cols([[1, 2], [1, 2], [2, 3], [3, 4], [4, 5], [5, 6]])
    delta = cols([[5, 6], [1, 2], [3, 4], [2, 3], [4, 5]])
    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, full, delta)
    summary = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store).run(store)
    st = oracle.Store()
    st.insert_static(0, (e0, e1))
    st.insert_recursive(1, full, delta)
    it, new = st.run_scc([1], [oracle.tc_rule(1, 0)])
    assert summary.iterations == it and summary.total_new_rows == new
    assert pairs(store.full(1)) == pairs(st.full(1))


def test_join_on_second_column_and_right_projection(cuda):
    # A rule keyed on the right relation's second column, projecting (R.0, L.1):
    # p(z, y) :- p(x, y), e(z, x). Exercises the sorted (key, row) index path.
    from sparkalog_b200.relational import (BinaryEqualityJoin, JoinInput, JoinProjection, RecursiveRulePlan,
                                           RecursiveSccPlan)

    R = rec()
    src, dst = generators.er_edges(3000, 3300, 21)
    e0, e1 = oracle.btree_pairs(src, dst)
    join = BinaryEqualityJoin(0, 1, (JoinProjection(JoinInput.RIGHT, 0), JoinProjection(JoinInput.LEFT, 1)))
    plan = RecursiveSccPlan([_rid(1)], [RecursiveRulePlan(_rid(1), _rid(1), _rid(0), join)])
    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    summary = R.RecursiveExecutor.compile(plan, store).run(store)
    st = oracle.Store()
    st.insert_static(0, (e0, e1))
    st.insert_recursive(1, (e0, e1), (e0, e1))
    it, new = st.run_scc([1], [oracle.rule_plan(1, 1, 0, left_key=0, right_key=1, projection=((1, 0), (0, 1)))])
    assert summary.iterations == it and summary.total_new_rows == new
    assert pairs(store.full(1)) == pairs(st.full(1))


def test_execute_binary_source_program(cuda, known_answers):
    # subset.rs:475-497 (value ids interned by first appearance).
    from sparkalog_b200.datalog import BinaryProgramPlan, BinarySccPlan, BinarySeedPlan, execute_binary
    from sparkalog_b200.recursion import transitive_closure_scc

    case = known_answers["source_program"]
    vid = {int(k): v for k, v in case["value_ids"].items()}
    edge, path = _rid(0), _rid(1)
    plan = BinaryProgramPlan(
        predicate_count=2,
        facts=[(edge, (vid[a], vid[b])) for a, b in [(1, 2), (2, 3), (3, 4)]],
        recursive_sccs=[BinarySccPlan(transitive_closure_scc(path, edge), [BinarySeedPlan(path, edge, (0, 1))])],
        outputs=[path],
    )
    result = execute_binary(plan, 16)
    assert result.summaries[0].iterations == case["iterations"]
    assert pairs(result.store.full(1)) == case["path_value_ids"]


def test_device_inputs_and_reads(cuda):
    R = rec()
    torch = cuda
    src, dst = generators.er_edges(20_000, 17_500, 3)
    d0 = torch.from_numpy(src.view(np.int32)).cuda()
    d1 = torch.from_numpy(dst.view(np.int32)).cuda()
    store = R.RelationStore()
    store.insert_static(0, (d0, d1))
    store.insert_recursive(1, (d0, d1), (d0, d1))
    R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store).run(store)
    n = store.rows(1)
    o0 = torch.empty(n, dtype=torch.int32, device="cuda")
    o1 = torch.empty(n, dtype=torch.int32, device="cuda")
    store.read_into(1, R.FULL, o0, o1)
    (w0, w1), _, _ = oracle.transitive_closure(src, dst, threads=8)
    assert np.array_equal(o0.cpu().numpy().view(np.uint32), w0)
    assert np.array_equal(o1.cpu().numpy().view(np.uint32), w1)


def _tc_with_stats(e0, e1, rule=None, oracle_rule=None, member=False):
    R = rec()
    from sparkalog_b200.relational import RecursiveSccPlan

    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    plan = R.transitive_closure_scc(_rid(1), _rid(0)) if rule is None else RecursiveSccPlan([_rid(1)], [rule])
    ex = R.RecursiveExecutor.compile(plan, store)
    ex.set_member_set(member)
    ex.set_profiling(True)
    summary = ex.run(store, 10_000)
    stats = ex.stats()
    st = oracle.Store()
    st.insert_static(0, (e0, e1))
    st.insert_recursive(1, (e0, e1), (e0, e1))
    it, new = st.run_scc([1], [oracle_rule or oracle.tc_rule(1, 0)])
    assert summary.iterations == it and summary.total_new_rows == new
    assert pairs(store.full(1)) == pairs(st.full(1))
    return stats


def test_fused_join_distinct_only_on_sparse_chain(cuda):
    # Every round of a chain fits the fused kernel's tiles: no general join.
    src = np.arange(700, dtype=np.uint32)
    stats = _tc_with_stats(src, src + 1)
    assert stats["classes"]["join_distinct"]["launches"] == stats["rounds"]
    assert stats["classes"]["join"]["launches"] == 0


def test_fused_join_distinct_falls_back_on_hub(cuda):
    # Node 0 reaches 6000 nodes in one step and a chain hangs off them, so its
    # x-run outgrows a fused tile: those rounds redo on the general kernels and
    # the result stays exact.
    hub = np.zeros(6000, dtype=np.uint32), np.arange(1, 6001, dtype=np.uint32)
    chain = np.arange(1, 400, dtype=np.uint32)
    er0, er1 = generators.er_edges(8000, 6000, 13)
    e0, e1 = oracle.btree_pairs(np.concatenate([hub[0], chain, er0]), np.concatenate([hub[1], chain + 1, er1]))
    stats = _tc_with_stats(e0, e1)
    assert stats["classes"]["join_distinct"]["launches"] > 0
    assert stats["classes"]["join"]["launches"] > 0


@pytest.mark.parametrize("fan", [150, 300, 700])
def test_fused_join_distinct_x_runs_past_the_window(cuda, fan):
    # Hubs whose x-runs in DELTA are longer than the rows a tile's window
    # reaches past its nominal end but fit a tile: the tile boundary is found
    # by the scan beyond the window and the rows are reloaded, exactly.
    hubs = np.repeat(np.array([0, 9000, 20000], dtype=np.uint32), fan)
    targets = np.concatenate([np.arange(1, fan + 1), np.arange(9001, 9001 + fan),
                              np.arange(20001, 20001 + fan)]).astype(np.uint32)
    er0, er1 = generators.er_edges(30000, 24000, 29)
    e0, e1 = oracle.btree_pairs(np.concatenate([hubs, er0]), np.concatenate([targets, er1]))
    stats = _tc_with_stats(e0, e1)
    assert stats["classes"]["join_distinct"]["launches"] > 0


def test_fused_join_distinct_join_on_first_column(cuda):
    # p(x, y) :- p(x, z), e(x, y): the join key is DELTA's first column.
    from sparkalog_b200.relational import BinaryEqualityJoin, JoinInput, JoinProjection, RecursiveRulePlan

    src, dst = generators.er_edges(4000, 6000, 17)
    e0, e1 = oracle.btree_pairs(src, dst)
    join = BinaryEqualityJoin(0, 0, (JoinProjection(JoinInput.LEFT, 0), JoinProjection(JoinInput.RIGHT, 1)))
    rule = RecursiveRulePlan(_rid(1), _rid(1), _rid(0), join)
    stats = _tc_with_stats(e0, e1, rule,
                           oracle.rule_plan(1, 1, 0, left_key=0, right_key=0, projection=((0, 0), (1, 1))))
    assert stats["classes"]["join_distinct"]["launches"] > 0


def test_fused_join_distinct_projects_delta_columns(cuda):
    # p(x, y) :- p(x, y), e(y, z): the output is DELTA itself, nothing new.
    from sparkalog_b200.relational import BinaryEqualityJoin, JoinInput, JoinProjection, RecursiveRulePlan

    src, dst = generators.er_edges(3000, 4000, 19)
    e0, e1 = oracle.btree_pairs(src, dst)
    join = BinaryEqualityJoin(1, 0, (JoinProjection(JoinInput.LEFT, 0), JoinProjection(JoinInput.LEFT, 1)))
    rule = RecursiveRulePlan(_rid(1), _rid(1), _rid(0), join)
    _tc_with_stats(e0, e1, rule, oracle.rule_plan(1, 1, 0, left_key=1, right_key=0, projection=((0, 0), (0, 1))))


@pytest.mark.parametrize("n,e,seed", [(2000, 8000, 1), (50_000, 60_000, 4), (300_000, 262_500, 6)])
def test_fused_and_general_rounds_agree(cuda, n, e, seed):
    # The fused join + distinct kernel and the general join / radix sort give
    # the same FULL, iteration count and new-row count (dense graphs also
    # exercise tile overflow and the smaller tiles that follow it).
    R = rec()
    src, dst = generators.er_edges(n, e, seed)
    e0, e1 = oracle.btree_pairs(src, dst)
    out = []
    for fused in (True, False):
        store = R.RelationStore()
        store.insert_static(0, (e0, e1))
        store.insert_recursive(1, (e0, e1), (e0, e1))
        ex = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store)
        ex.set_fused(fused)
        ex.set_profiling(True)
        summary = ex.run(store, 10_000)
        stats = ex.stats()
        assert (stats["classes"]["join_distinct"]["launches"] > 0) == fused
        f0, f1 = store.full(1)
        out.append((summary.iterations, summary.total_new_rows, f0, f1))
    assert out[0][:2] == out[1][:2]
    assert np.array_equal(out[0][2], out[1][2]) and np.array_equal(out[0][3], out[1][3])


def test_fused_join_distinct_through_sorted_index(cuda):
    # p(x, z) :- p(x, y), e(z, y): the right relation is indexed on its second
    # column, so the fused kernel gathers right rows through the index's row ids.
    from sparkalog_b200.relational import BinaryEqualityJoin, JoinInput, JoinProjection, RecursiveRulePlan

    src, dst = generators.er_edges(5000, 5200, 23)
    e0, e1 = oracle.btree_pairs(src, dst)
    join = BinaryEqualityJoin(1, 1, (JoinProjection(JoinInput.LEFT, 0), JoinProjection(JoinInput.RIGHT, 0)))
    rule = RecursiveRulePlan(_rid(1), _rid(1), _rid(0), join)
    stats = _tc_with_stats(e0, e1, rule,
                           oracle.rule_plan(1, 1, 0, left_key=1, right_key=1, projection=((0, 0), (1, 0))))
    assert stats["classes"]["join_distinct"]["launches"] > 0


@pytest.mark.parametrize("n,e,seed", [(2000, 8000, 1), (60_000, 55_000, 8), (300_000, 262_500, 6)])
def test_member_set_and_level_search_agree(cuda, n, e, seed):
    # FULL's hash set and the directory search of the sorted levels give the
    # same fixpoint (the set is rebuilt larger several times as FULL grows).
    R = rec()
    src, dst = generators.er_edges(n, e, seed)
    e0, e1 = oracle.btree_pairs(src, dst)
    out = []
    for member in (True, False):
        store = R.RelationStore()
        store.insert_static(0, (e0, e1))
        store.insert_recursive(1, (e0, e1), (e0, e1))
        ex = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store)
        ex.set_member_set(member)
        summary = ex.run(store, 10_000)
        out.append((summary.iterations, summary.total_new_rows) + store.full(1))
    assert out[0][:2] == out[1][:2]
    assert np.array_equal(out[0][2], out[1][2]) and np.array_equal(out[0][3], out[1][3])


def test_member_set_holds_the_all_ones_row(cuda):
    # The row (0xffffffff, 0xffffffff) equals the hash set's empty-slot marker
    # and is tracked apart from the slots.
    top = 0xFFFFFFFF
    pairs_in = [[1, top], [top, top], [top, 2], [2, 3], [3, 1]]
    e0, e1 = oracle.btree_pairs(*cols(pairs_in))
    _tc_with_stats(e0, e1, member=True)
    _tc_with_stats(e0, e1, member=False)


def test_member_set_follows_appends(cuda):
    # A resident fixpoint continued after store.append: the appended rows go
    # into FULL's hash set, and the closure equals a fresh run from the union.
    R = rec()
    src, dst = generators.er_edges(20_000, 16_000, 31)
    e0, e1 = oracle.btree_pairs(src, dst)
    extra0, extra1 = generators.uniform_pairs(20_000, 3_000, 32)
    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    ex = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store)
    ex.set_member_set(True)
    ex.run(store, 10_000)
    store.append(1, (extra0, extra1))
    ex.run(store, 10_000)
    s0, s1 = oracle.btree_pairs(np.concatenate([e0, extra0]), np.concatenate([e1, extra1]))
    st = oracle.Store()
    st.insert_static(0, (e0, e1))
    st.insert_recursive(1, (s0, s1), (s0, s1))
    st.run_scc([1], [oracle.tc_rule(1, 0)])
    assert pairs(store.full(1)) == pairs(st.full(1))


@pytest.mark.parametrize("fused", [True, False])
def test_round_trace_cardinalities(cuda, fused):
    # Per-round operator cardinalities against a plain semi-naive loop in
    # Python: |DELTA|, |join|, |distinct|, |NEWT| and |FULL| after the round.
    R = rec()
    src, dst = generators.er_edges(1500, 1900, 41)
    e0, e1 = oracle.btree_pairs(src, dst)
    adj = {}
    for a, b in zip(e0.tolist(), e1.tolist()):
        adj.setdefault(a, []).append(b)
    full = set(zip(e0.tolist(), e1.tolist()))
    delta = sorted(full)
    expect = []
    while delta:
        joined = [(x, z) for x, y in delta for z in adj.get(y, ())]
        unique = set(joined)
        new = unique - full
        full |= new
        expect.append((len(delta), len(joined), len(unique), len(new), len(full)))
        delta = sorted(new)
    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    ex = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store)
    ex.set_fused(fused)
    summary = ex.run(store, 10_000)
    got = [(r["delta_rows"], r["join_rows"], r["unique_rows"], r["new_rows"], r["full_rows"]) for r in ex.trace()]
    assert summary.iterations == len(expect)
    assert got == expect
    assert [r["round"] for r in ex.trace(reset=True)] == list(range(1, len(expect) + 1))
    assert ex.trace() == []


def _run_tc(src, dst, tuning=None, device_loop=True, steps=None):
    R = rec()
    e0, e1 = oracle.btree_pairs(src, dst)
    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    ex = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store)
    if tuning:
        ex.set_tuning(tuning)
    ex.set_device_loop(device_loop)
    if steps is None:
        summary = ex.run(store)
        iterations, new = summary.iterations, summary.total_new_rows
    else:
        iterations = new = 0
        while True:
            summary, done = ex.step(store, steps)
            iterations += summary.iterations
            new += summary.total_new_rows
            if done:
                break
    trace = ex.trace()
    loop = ex.device_loop_stats()
    full = store.full(1)
    ex.close()
    store.close()
    return full, iterations, new, trace, loop


TUNINGS = [
    {},
    {"merge_items": 7, "levels": 4, "dir_rows_log2": 2, "group_lanes": 4},
    {"merge_items": 15, "levels": 2, "dir_rows_log2": 0, "group_lanes": 16, "group_candidates": 1 << 21},
    {"level_ratio": 2, "sparse_candidates": 1 << 22, "group_candidates": 1 << 12, "fused_rows_cap": 128},
    {"bloom_bits": 8},
    {"bloom_bits": 4, "levels": 4, "group_candidates": 1 << 12},
    {"merge_anti_ratio": 0, "sparse_items": 2, "levels": 4, "group_candidates": 1 << 10},
    {"sparse_items": 3, "group_candidates": 1 << 10},
    {"compact_index": 0},
    {"merge_anti_ratio": 1024, "levels": 4, "level_ratio": 2},
    {"merge_anti_ratio": 1024, "levels": 2, "group_candidates": 1 << 10, "sparse_candidates": 1 << 12},
]


@pytest.mark.parametrize("tuning", TUNINGS)
def test_every_tuning_gives_the_oracle_fixpoint(cuda, tuning):
    # Launch shapes, directory granularity, level count and thresholds change
    # speed only: FULL, iteration count and the per-round trace are the same.
    src, dst = generators.er_edges(300_000, 262_500, 6)
    (w0, w1), it, new = oracle.transitive_closure(src, dst, threads=8)
    full, iterations, derived, trace, _ = _run_tc(src, dst, tuning)
    base = _run_tc(src, dst, None, device_loop=False)
    assert iterations == it and derived == new
    assert np.array_equal(full[0], w0) and np.array_equal(full[1], w1)
    assert [(r["delta_rows"], r["unique_rows"], r["new_rows"], r["full_rows"]) for r in trace] == \
        [(r["delta_rows"], r["unique_rows"], r["new_rows"], r["full_rows"]) for r in base[3]]


@pytest.mark.parametrize("n,e,seed", [(300_000, 262_500, 6), (1_000_000, 875_000, 8), (5000, 4500, 2)])
def test_device_loop_matches_host_loop(cuda, n, e, seed):
    # The tail rounds run as a CUDA graph WHILE loop with a device-side
    # convergence test; FULL, iterations and every round's cardinalities equal
    # the host-driven loop's, and the loop really ran.
    src, dst = generators.er_edges(n, e, seed)
    on = _run_tc(src, dst, None, device_loop=True)
    off = _run_tc(src, dst, None, device_loop=False)
    assert on[1] == off[1] and on[2] == off[2]
    assert np.array_equal(on[0][0], off[0][0]) and np.array_equal(on[0][1], off[0][1])
    assert on[3] == off[3]
    assert off[4] == (0, 0)
    if n >= 300_000:
        launches, rounds = on[4]
        assert launches >= 1 and rounds >= 10


def test_device_loop_respects_step_limits(cuda):
    # executor_step with a few rounds at a time: the device loop stops at each
    # step's limit and resumes, with the same result.
    src, dst = generators.er_edges(300_000, 262_500, 6)
    (w0, w1), it, new = oracle.transitive_closure(src, dst, threads=8)
    full, iterations, derived, _, loop = _run_tc(src, dst, None, device_loop=True, steps=3)
    assert iterations == it and derived == new
    assert np.array_equal(full[0], w0) and np.array_equal(full[1], w1)


@pytest.mark.parametrize("levels", [2, 3, 4])
def test_compact_merges_full_into_one_sorted_run(cuda, levels):
    # store.compact merges FULL's levels (smallest first) into one sorted run:
    # the rows, and what a later read returns, are the oracle's fixpoint.
    src, dst = generators.er_edges(300_000, 262_500, 6)
    (w0, w1), it, new = oracle.transitive_closure(src, dst, threads=8)
    R = rec()
    e0, e1 = oracle.btree_pairs(src, dst)
    store = R.RelationStore()
    store.insert_static(0, (e0, e1))
    store.insert_recursive(1, (e0, e1), (e0, e1))
    ex = R.RecursiveExecutor.compile(R.transitive_closure_scc(_rid(1), _rid(0)), store)
    ex.set_tuning({"levels": levels})
    summary = ex.run(store)
    assert summary.iterations == it and summary.total_new_rows == new
    store.compact(1)
    assert store.rows(1) == len(w0)
    store.compact(1)  # already one run: nothing to merge
    f0, f1 = store.full(1)
    assert np.array_equal(f0, w0) and np.array_equal(f1, w1)
    ex.close()
    store.close()
