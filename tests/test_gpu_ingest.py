"""GPU parsing of binary u32 relations (load_binary_u32, crates/sparkalog-storage/src/io.rs:72-138)
against the oracle's line-by-line restatement: rows bit-exact, errors with the same kind, line
and column."""

import numpy as np
import pytest

import oracle
from conftest import pairs

pytestmark = pytest.mark.gpu


def rec():
    from sparkalog_b200 import recursion

    return recursion


def load(text, **kw):
    R = rec()
    store = R.RelationStore()
    n = store.load_binary_u32(0, text, **kw)
    return store, n


def test_load_known_answers_and_syntax(cuda, known_answers):
    R = rec()
    for case in known_answers["load_binary_u32"]:
        if "error" in case:
            with pytest.raises(R.LoadError) as e:
                load(case["text"])
            assert e.value.kind == case["error"]
            if "line" in case:
                assert e.value.line == case["line"]
        else:
            store, n = load(case["text"])
            assert n == len(case["first"])
            f, s = store.full(0)
            assert sorted(zip(f.tolist(), s.tolist())) == sorted(zip(case["first"], case["second"]))
    store, n = load(b"+7 007\r\n  \t8\t9  \n4294967295 0")
    assert n == 3 and pairs(store.full(0)) == [[7, 7], [8, 9], [4294967295, 0]]
    for text, kind, line, column, value in [(b"1 2\n1 -2\n", "InvalidU32", 2, 2, "-2"),
                                             (b"1 4294967296\n", "InvalidU32", 1, 2, "4294967296"),
                                             (b"x 1\n", "InvalidU32", 1, 1, "x"),
                                             (b"1\n", "InvalidFieldCount", 1, 0, None),
                                             (b"1 2\n3 + \n", "InvalidU32", 2, 2, "+")]:
        with pytest.raises(R.LoadError) as e:
            load(text)
        assert (e.value.kind, e.value.line, e.value.value) == (kind, line, value)
        if kind == "InvalidU32":
            assert e.value.column == column
    store, n = load(b"")
    assert n == 0 and store.rows(0) == 0


def test_load_error_precedence(cuda):
    # The first failing line wins, and a Git LFS pointer anywhere wins over
    # field errors (count_rows reads the whole text before populate_columns).
    R = rec()
    lines = [f"{i} {i + 1}" for i in range(10_000)]
    lines[7000] = "7000 x"
    lines[3000] = "3000"
    with pytest.raises(R.LoadError) as e:
        load("\n".join(lines))
    assert (e.value.kind, e.value.line) == ("InvalidFieldCount", 3001)
    lines.append("version https://git-lfs.github.com/spec/v1")
    with pytest.raises(R.LoadError) as e:
        load("\n".join(lines))
    assert e.value.kind == "GitLfsPointer"


def test_load_random_text_matches_oracle_and_runs(cuda):
    # Two million lines with comments, blank lines, CRLF endings, tabs and
    # '+' signs, read on the GPU, equal the oracle's columns in file order;
    # loaded as the seed of a fixpoint, the closure equals the oracle's.
    R = rec()
    torch = cuda
    rng = np.random.default_rng(11)
    n = 2_000_000
    a = rng.integers(0, 1 << 32, size=n, dtype=np.uint64)
    b = rng.integers(0, 1 << 32, size=n, dtype=np.uint64)
    kinds = rng.integers(0, 20, size=n)
    out = []
    for i in range(n):
        k = kinds[i]
        if k == 0:
            out.append("# comment")
        elif k == 1:
            out.append("   ")
        elif k == 2:
            out.append(f"\t{a[i]}\t+{b[i]}\r")
        elif k == 3:
            out.append("% x y z")
        else:
            out.append(f"{a[i]} {b[i]}")
    text = ("\n".join(out) + "\n").encode()
    want = oracle.load_binary_u32(text)
    store = R.RelationStore()
    got_n = store.load_binary_u32(0, torch.from_numpy(np.frombuffer(text, dtype=np.uint8).copy()).cuda())
    assert got_n == len(want[0])
    # A static relation keeps its rows as read, in file order.
    f, s = store.full(0)
    assert np.array_equal(f, want[0]) and np.array_equal(s, want[1])
    small = b"1 2\n2 3\n# c\n3 4\n\n4 5\n"
    store2 = R.RelationStore()
    store2.load_binary_u32(0, small)
    store2.load_binary_u32(1, small, recursive=True)
    from sparkalog_b200.relational import RelationId

    R.RecursiveExecutor.compile(R.transitive_closure_scc(RelationId(1), RelationId(0)), store2).run(store2)
    assert pairs(store2.full(1)) == [[1, 2], [1, 3], [1, 4], [1, 5], [2, 3], [2, 4], [2, 5], [3, 4], [3, 5], [4, 5]]


# ---------------------------------------------------------------------------
# load_delimited (database.rs:165-177, ingest.rs:20-120) for u32 relations.
# ---------------------------------------------------------------------------
def load_delimited(text, **kw):
    R = rec()
    store = R.RelationStore()
    n = store.load_delimited_u32(0, text, **kw)
    return store, n


def oracle_rows(text, delimiter=",", has_header=False):
    rows = oracle.parse_delimited(text, delimiter, has_header)
    assert all(len(r) == 2 and r[0][0] == "u32" and r[1][0] == "u32" for r in rows)
    return [[r[0][1], r[1][1]] for r in rows]


def test_load_delimited_known_answers(cuda, known_answers):
    R = rec()
    for case in known_answers["load_delimited"]:
        text = case.get("text")
        if text is None:
            text = "\n".join(case["format"].format(v=v) for v in range(case["generated_rows"]))
        rows = oracle.parse_delimited(text, case["delimiter"], case["has_header"])
        if all(len(r) == 2 and r[0][0] == r[1][0] == "u32" for r in rows):
            store, n = load_delimited(text, delimiter=case["delimiter"], has_header=case["has_header"])
            assert n == case.get("rows", len(rows))
            f, s = store.full(0)
            assert sorted(zip(f.tolist(), s.tolist())) == sorted((r[0][1], r[1][1]) for r in rows)
        else:
            # Strings and symbols: this entry point loads u32 relations only.
            with pytest.raises(R.LoadError) as e:
                load_delimited(text, delimiter=case["delimiter"], has_header=case["has_header"])
            assert e.value.kind in ("NotU32", "Arity")
    # The CSV of ingest.rs:145-150: 'alpha' (line 2, byte column 3) is a symbol.
    with pytest.raises(R.LoadError) as e:
        load_delimited('from,to\n1,alpha\n2,"a string"\n', has_header=True)
    assert (e.value.kind, e.value.line, e.value.column, e.value.value) == ("NotU32", 2, 3, "alpha")


def test_load_delimited_against_oracle(cuda):
    rng = np.random.default_rng(31)
    n = 20_000
    a = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    b = rng.integers(0, 1000, n, dtype=np.uint64)
    pads = [" ", "\t", " ", "　", "", "  "]
    ends = ["\n", "\r\n"]
    lines = ["src,dst"]
    for i in range(n):
        p, q = pads[i % len(pads)], pads[(i // 7) % len(pads)]
        sign = "+" if i % 11 == 0 else ""
        lines.append(f"{p}{sign}{a[i]}{q},{q}{b[i]}{p}" + ends[i % 2].rstrip("\n"))
        if i % 97 == 0:
            lines.append(" \t ")  # blank: skipped
    text = "\n".join(lines) + "\n"
    want = oracle_rows(text, ",", True)
    store, rows = load_delimited(text, has_header=True)
    assert rows == len(want) == n
    assert pairs(store.full(0)) == want  # a static relation keeps file order
    # Tab-separated, no header, no final newline, from a device buffer.
    import torch

    tsv = "\n".join(f"{x}\t{y}" for x, y in zip(a[:500].tolist(), b[:500].tolist()))
    dev = torch.from_numpy(np.frombuffer(tsv.encode(), dtype=np.uint8).copy()).cuda()
    store, rows = load_delimited(dev, delimiter="\t")
    assert rows == 500 and pairs(store.full(0)) == oracle_rows(tsv, "\t")
    # Interning the rows in order gives load_delimited's value ids.
    from sparkalog_b200.datalog import ValueCatalog

    text = "".join(f"{x},{y}\n" for x, y in zip(b[:300].tolist(), b[300:600].tolist()))
    store, _ = load_delimited(text)
    f, s = store.full(0)
    want_ids, _ = oracle.load_delimited(text, 2)
    got = ValueCatalog().intern_rows(torch.from_numpy(f.view(np.int32)).cuda(), torch.from_numpy(s.view(np.int32)).cuda())
    assert np.array_equal(torch.stack(got, dim=1).cpu().numpy().view(np.uint32), want_ids)


def test_load_delimited_errors(cuda):
    R = rec()
    # Syntax errors: the reference's line, byte column and message.
    for text in ["1,2\n3,", '1,2\n"ab,3\n', '1,2\n"a"b,1\n', "1,2\n1,,2\n", "x,y\n\n 1 , \n", "4,5\r\n6,\r\n"]:
        with pytest.raises(oracle.OracleDelimitedError) as want:
            oracle.parse_delimited(text)
        with pytest.raises(R.LoadError) as got:
            load_delimited(text)
        assert (got.value.line, got.value.column, got.value.kind) == (want.value.line, want.value.column,
                                                                      want.value.message), text
    # A syntax error anywhere comes before an earlier non-u32 row.
    with pytest.raises(R.LoadError) as e:
        load_delimited("1,x\n2,3\n4,\n")
    assert (e.value.kind, e.value.line) == ("record ends with an empty field", 3)
    # Rows that parse but are not two u32 values.
    for text, kind, line, column, value in [("1,2\n3,4,5\n", "Arity", 2, 3, None),
                                             ("1,2\n7\n", "Arity", 2, 1, None),
                                             ('1,2\n3,"q"\n', "NotU32", 2, 3, '"q"'),
                                             ("1,2\n3, -4\n", "NotU32", 2, 3, "-4"),
                                             ("1,4294967296\n", "NotU32", 1, 3, "4294967296")]:
        with pytest.raises(R.LoadError) as e:
            load_delimited(text)
        assert (e.value.kind, e.value.line, e.value.column, e.value.value) == (kind, line, column, value), text
    # Whitespace delimiters other than tab are refused (ingest.rs:24-30).
    with pytest.raises(R.GenericExecutionError):
        load_delimited("1 2\n", delimiter=" ")
    store, n = load_delimited("")
    assert n == 0 and store.rows(0) == 0
    store, n = load_delimited("a,b\n", has_header=True)
    assert n == 0
