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
