"""CPU tests: the oracle pinned against the reference's own known answers.

The oracle is only trusted for parity once it reproduces every known-answer
vector of the reference's tests (tests/golden/known_answers.json) and the
serial/parallel equalities the reference asserts for each operator.
"""

import numpy as np
import pytest

import oracle
from conftest import cols, pairs
from sparkalog_b200 import generators


def test_distinct_known_answers(known_answers):
    for case in known_answers["distinct"]:
        for threads in (1, 4):
            assert pairs(oracle.distinct(cols(case["input"]), threads=threads)) == case["expected"], case["source"]


def test_anti_join_known_answers(known_answers):
    for case in known_answers["anti_join"]:
        for threads in (1, 4):
            got = oracle.anti_join(cols(case["left"]), cols(case["right"]), threads=threads)
            assert pairs(got) == case["expected"], case["source"]


def test_union_known_answers(known_answers):
    for case in known_answers["union"]:
        for threads in (1, 4):
            got = oracle.union(cols(case["left"]), cols(case["right"]), threads=threads)
            assert pairs(got) == case["expected"], case["source"]


def test_join_known_answers(known_answers):
    for case in known_answers["join"]:
        proj = tuple(tuple(p) for p in case["projection"])
        for threads in (1, 4):
            got = oracle.join(cols(case["left"]), cols(case["right"]), case["left_key"], case["right_key"], proj,
                              threads=threads)
            assert pairs(got) == case["expected"], case["source"]


def run_fixpoint_case(case, threads=1):
    st = oracle.Store()
    for rid, rows in case["relations"].items():
        st.insert_static(int(rid), cols(rows))
    for rid, fd in case["recursive"].items():
        st.insert_recursive(int(rid), cols(fd["full"]), cols(fd["delta"]))
    rules = [oracle.rule_plan(r["target"], r["delta_input"], r["right_input"]) for r in case["rules"]]
    it, new = st.run_scc(case["scc"], rules, 16, threads)
    return st, it, new


def test_fixpoint_known_answers(known_answers):
    for case in known_answers["fixpoint"]:
        for threads in (1, 3):
            st, it, new = run_fixpoint_case(case, threads)
            if "iterations" in case:
                assert it == case["iterations"], case["source"]
            if "total_new_rows" in case:
                assert new == case["total_new_rows"], case["source"]
            for rid, rows in case["full"].items():
                assert pairs(st.full(int(rid))) == rows, case["source"]
                assert len(st.delta(int(rid))[0]) == 0


def test_incompatible_plans_rejected():
    # generic.rs:917-946
    st = oracle.Store()
    st.insert_static(0, cols([[1, 2]]))
    st.insert_recursive(1, cols([[1, 2]]), cols([[1, 2]]))
    first = oracle.tc_rule(1, 0)
    bad = oracle.rule_plan(1, 1, 0, union_cols=((0, 1), (1, 0)))
    with pytest.raises(oracle.OracleError) as err:
        st.run_scc([1], [first, bad])
    assert err.value.code == -8


def test_iteration_limit():
    st = oracle.Store()
    edges = cols([[i, i + 1] for i in range(10)])
    st.insert_static(0, edges)
    st.insert_recursive(1, edges, edges)
    with pytest.raises(oracle.OracleError) as err:
        st.run_scc([1], [oracle.tc_rule(1, 0)], max_iterations=3)
    assert err.value.code == -10


@pytest.mark.parametrize("n", [2, 3, 17, 128])
def test_chain_closure_size(n):
    # tc-fixpoint.rs:142-144: a chain of n vertices closes to n(n-1)/2 rows.
    src = np.arange(n - 1, dtype=np.uint32)
    (p0, p1), it, new = oracle.transitive_closure(src, src + 1)
    assert len(p0) == n * (n - 1) // 2
    assert it == n - 1


def test_source_program_value_ids(known_answers):
    # subset.rs:475-497 through execute_binary, with the catalog's
    # first-appearance interning (1 -> 0, 2 -> 1, ...).
    case = known_answers["source_program"]
    vid = {int(k): v for k, v in case["value_ids"].items()}
    edge, path = 0, 1
    facts = [(edge, (vid[a], vid[b])) for a, b in [(1, 2), (2, 3), (3, 4)]]
    scc = oracle.SccPlan([path], [oracle.tc_rule(path, edge)], [oracle.SeedPlan(path, edge, (0, 1))])
    st, summaries = oracle.execute_binary(2, facts, [scc])
    assert summaries[0][0] == case["iterations"]
    assert pairs(st.full(path)) == case["path_value_ids"]


def test_general_cpu_negation(known_answers):
    # general.rs:673-690: node(a,b,c), flag(b, yes), blocked(x) :- flag(x, yes),
    # allowed(x) :- node(x), !blocked(x). Values interned a=0, b=1, c=2, yes=3;
    # relations node=0, flag=1, blocked=2, allowed=3.
    case = known_answers["negation"]
    facts = [(0, (0,)), (0, (1,)), (0, (2,)), (1, (1, 3))]
    blocked = oracle.Clause(2, [("b", 0)], [oracle.Atom(1, [("b", 0), ("v", 3)])])
    allowed = oracle.Clause(3, [("b", 0)], [oracle.Atom(0, [("b", 0)])], [oracle.Atom(2, [("b", 0)])])
    strata = [[oracle.GeneralScc([2], False, [blocked], [])], [oracle.GeneralScc([3], False, [allowed], [])]]
    full, summaries = oracle.general_cpu(4, facts, strata)
    assert len(strata) == case["strata"]
    assert len(full[2]) == case["blocked_rows"]
    assert len(full[3]) == case["allowed_rows"]
    assert summaries[0][1] == 1 and summaries[1][1] == 1


def test_general_cpu_matches_binary_tc():
    # The nested-loop GeneralCpu evaluation and the operator pipeline agree on
    # a small random TC (iteration count included).
    src, dst = generators.er_edges(40, 60, 9)
    (p0, p1), it, new = oracle.transitive_closure(src, dst)
    facts = [(0, (int(a), int(b))) for a, b in zip(src, dst)]
    seed = oracle.Clause(1, [("b", 0), ("b", 1)], [oracle.Atom(0, [("b", 0), ("b", 1)])])
    rec = oracle.Clause(1, [("b", 0), ("b", 2)], [oracle.Atom(1, [("b", 0), ("b", 1)], delta=True),
                                                   oracle.Atom(0, [("b", 1), ("b", 2)])])
    full, summaries = oracle.general_cpu(2, facts, [[oracle.GeneralScc([1], True, [seed], [rec])]])
    assert sorted(full[1]) == [tuple(p) for p in pairs((p0, p1))]
    assert summaries[0][1] == it
    assert summaries[0][2] == new


def test_negation_pipeline_matches_general_cpu():
    # Stratified negation unreached(x, y) :- cand(x, y), !path(x, y): the
    # anti-join of the deduplicated candidates against FULL(path) equals the
    # GeneralCpu evaluation.
    src, dst = generators.er_edges(30, 25, 4)
    (p0, p1), _, _ = oracle.transitive_closure(src, dst)
    c0, c1 = generators.uniform_pairs(30, 300, 8)
    got = oracle.anti_join(oracle.distinct((c0, c1)), (p0, p1))
    facts = [(2, (int(a), int(b))) for a, b in zip(c0, c1)] + [(1, (int(a), int(b))) for a, b in zip(p0, p1)]
    clause = oracle.Clause(3, [("b", 0), ("b", 1)], [oracle.Atom(2, [("b", 0), ("b", 1)])],
                           [oracle.Atom(1, [("b", 0), ("b", 1)])])
    full, _ = oracle.general_cpu(4, facts, [[oracle.GeneralScc([3], False, [clause], [])]])
    assert [tuple(p) for p in pairs(got)] == sorted(full[3])


@pytest.mark.parametrize("n,e,seed", [(2000, 8000, 1), (64, 500, 3), (100_000, 87_500, 11)])
def test_generators_agree_with_oracle(n, e, seed):
    a = generators.er_edges(n, e, seed)
    b = oracle.er_edges(n, e, seed)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert len(a[0]) == e
    assert not np.any(a[0] == a[1])


def test_parallel_operators_match_serial():
    rng = np.random.default_rng(5)
    a = rng.integers(0, 300, size=(20_000, 2)).astype(np.uint32)
    b = rng.integers(0, 300, size=(15_000, 2)).astype(np.uint32)
    da = oracle.distinct((a[:, 0], a[:, 1]))
    db = oracle.distinct((b[:, 0], b[:, 1]))
    for f in (oracle.anti_join, oracle.union):
        assert pairs(f(da, db, threads=1)) == pairs(f(da, db, threads=6))
    assert pairs(oracle.distinct((a[:, 0], a[:, 1]), threads=6)) == pairs(da)
    j1 = oracle.join(da, db, threads=1)
    j6 = oracle.join(da, db, threads=6)
    assert pairs(j1) == pairs(j6)


def test_filter_known_answers(known_answers):
    # lib.rs:2015-2027, 2403-2445: every predicate, serial == parallel, empty columns.
    for case in known_answers["filter"]:
        if "values_mod" in case:
            n, m = case["values_mod"]
            values = np.arange(n, dtype=np.uint32) % m
            a = oracle.filter_serial(values, case["op"], case["operand"])
            b = oracle.filter_parallel(values, case["op"], case["operand"])
            assert len(a) == case["expected_count"] and np.array_equal(a, b)
            continue
        for op, operand, want in case["cases"]:
            assert oracle.filter_serial(case["values"], op, operand).tolist() == want, case["source"]
            assert oracle.filter_parallel(case["values"], op, operand).tolist() == want, case["source"]
    assert oracle.filter_serial([1, 2, 3], 9, 1).tolist() == []  # unknown operation code: no rows


def test_load_binary_u32_known_answers(known_answers):
    # io.rs:145-174, plus the u32 syntax of str::parse and the line rules.
    for case in known_answers["load_binary_u32"]:
        if "error" in case:
            with pytest.raises(oracle.OracleLoadError) as e:
                oracle.load_binary_u32(case["text"].encode())
            assert e.value.kind == case["error"] and e.value.line == case.get("line", 0)
        else:
            f, s = oracle.load_binary_u32(case["text"].encode())
            assert f.tolist() == case["first"] and s.tolist() == case["second"]
    f, s = oracle.load_binary_u32(b"+7 007\r\n  \t8\t9  \n4294967295 0")
    assert f.tolist() == [7, 8, 4294967295] and s.tolist() == [7, 9, 0]
    for text, kind, line, column in [(b"1 2\n1 -2\n", "InvalidU32", 2, 2), (b"1 4294967296\n", "InvalidU32", 1, 2),
                                      (b"x 1\n", "InvalidU32", 1, 1), (b"1\n", "InvalidFieldCount", 1, 0),
                                      (b"1 2\n3 + \n", "InvalidU32", 2, 2)]:
        with pytest.raises(oracle.OracleLoadError) as e:
            oracle.load_binary_u32(text)
        assert (e.value.kind, e.value.line, e.value.column) == (kind, line, column)


def test_load_and_intern_c_restatements_agree():
    # The C restatements (used for timing) equal the line-by-line Python ones.
    rng = np.random.default_rng(9)
    rows = rng.integers(0, 1 << 32, size=(20_000, 2), dtype=np.uint64)
    lines = [("# c" if i % 13 == 0 else f"{a}\t+{b}\r" if i % 7 == 0 else f"{a} {b}") for i, (a, b) in enumerate(rows)]
    text = "\n".join(lines).encode()
    a = oracle.load_binary_u32(text)
    b = oracle.load_binary_u32_c(text)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for bad in (b"1 2\n3 x\n", b"1 2 3\n", b"version https://git-lfs.github.com/spec/v1\n"):
        with pytest.raises(oracle.OracleLoadError) as e1:
            oracle.load_binary_u32(bad)
        with pytest.raises(oracle.OracleLoadError) as e2:
            oracle.load_binary_u32_c(bad)
        assert (e1.value.kind, e1.value.line, e1.value.column) == (e2.value.kind, e2.value.line, e2.value.column)
    v = rng.integers(0, 5000, size=50_000).astype(np.uint32)
    assert np.array_equal(oracle.intern(v)[0], oracle.intern_c(v))


def test_general_tc_c_restatement(known_answers):
    # GeneralCpu's nested loop (general.rs:393-536) in C: the chain of
    # generic.rs:716-746 and small ER graphs against the operator pipeline.
    r = oracle.general_tc_c(np.array([1, 2, 3, 4], np.uint32), np.array([2, 3, 4, 5], np.uint32))
    assert r["converged"] and r["rounds"] == 4 and r["new_rows"] == 6
    for nodes, edges, seed in [(300, 280, 5), (500, 900, 6)]:
        s, d = generators.er_edges(nodes, edges, seed)
        (_, _), it, new = oracle.transitive_closure(s, d)
        e0, _ = oracle.btree_pairs(s, d)
        r = oracle.general_tc_c(s, d)
        assert r["converged"] and r["rounds"] == it and r["new_rows"] == new
        # Every round tests (|edge| + 1) tuples per DELTA tuple: the figure the
        # bench extrapolates a capped sample by.
        assert r["tests"] == (len(e0) + 1) * (len(e0) + new)
    capped = oracle.general_tc_c(*generators.er_edges(2000, 8000, 1), time_cap_s=0.0)
    assert not capped["converged"] and capped["rounds"] == 0


def _value(v):
    return (v[0], v[1])


def test_load_delimited_known_answers(known_answers):
    # parse_delimited_parallel / Database::load_delimited vectors
    # (ingest.rs:143-181, database.rs:441-457).
    for case in known_answers["load_delimited"]:
        text = case.get("text")
        if text is None:
            text = "\n".join(case["format"].format(v=v) for v in range(case["generated_rows"]))
        rows = oracle.parse_delimited(text, case["delimiter"], case["has_header"])
        if "rows" in case:
            assert len(rows) == case["rows"], case["source"]
        for r, length in enumerate(case.get("row_lengths", [])):
            assert len(rows[r]) == length, case["source"]
        for r, c, want in case.get("checks", []):
            got = rows[r] if c is None else rows[r][c]
            want = [_value(v) for v in want] if c is None else _value(want)
            assert got == want, case["source"]
        if "arity" in case:
            ids, catalog = oracle.load_delimited(text, case["arity"], case["delimiter"], case["has_header"])
            # path(x, y) :- edge(x, y): the copy has the loaded rows.
            assert len({tuple(r) for r in ids.tolist()}) == case["path_rows"]


def test_load_delimited_errors_and_u32_subset():
    # Error positions follow parse_record (ingest.rs:43-120): 1-based line,
    # byte column; a whitespace delimiter other than tab is refused.
    cases = [("1,", (1, 2, "record ends with an empty field")), ('"ab', (1, 1, "unterminated quoted field")),
             ('"a"b,1', (1, 4, "expected delimiter after quoted field")),
             ("1,,2", (1, 3, "empty fields are not values")), ("x\n\n 1 , ", (3, 5, "empty fields are not values"))]
    for text, (line, column, message) in cases:
        with pytest.raises(oracle.OracleDelimitedError) as e:
            oracle.parse_delimited(text)
        assert (e.value.line, e.value.column, e.value.message) == (line, column, message), text
    with pytest.raises(oracle.OracleDelimitedError):
        oracle.parse_delimited("1 2", " ")
    # Quotes, trimming, CRLF, symbols that only look numeric, u32 overflow.
    rows = oracle.parse_delimited('"a ""q"" b", x \r\n+7,4294967296\r\n-1,007\n')
    assert rows == [[("string", 'a "q" b'), ("symbol", "x")], [("u32", 7), ("symbol", "4294967296")],
                    [("symbol", "-1"), ("u32", 7)]]
    with pytest.raises(oracle.OracleArityError):
        oracle.load_delimited("1,2,3\n", 2)
    # A u32-only file: the same rows and ids as load_binary_u32 + interning.
    src, dst = generators.er_edges(500, 700, 9)
    text = "".join(f"{a},{b}\n" for a, b in zip(src.tolist(), dst.tolist()))
    ids, _ = oracle.load_delimited(text, 2)
    f, s = oracle.load_binary_u32(text.replace(",", "\t").encode())
    want, _ = oracle.intern(np.stack([f, s], axis=1).reshape(-1))
    assert np.array_equal(ids.reshape(-1), want)
