"""GPU parity of mixed-value ingest and interning (U32, String, Symbol).

Database::load_delimited (crates/sparkalog-datalog/src/database.rs:165-177)
parses a delimited text (ingest.rs:20-120) and interns every value in row
order (ValueCatalog::intern, catalog.rs:108-117). The device loader
(sparkalog_store_load_delimited_values) must give every row the oracle's
value ids and leave the catalog holding the oracle's values in id order: the
reference's own vectors (ingest.rs:143-181), random files with quoted
strings ('""' escapes, UTF-8), symbols and numbers, two files into one
catalog, the U32 entry points on a mixed catalog, and the errors.
"""

import numpy as np
import pytest

import oracle
from conftest import pairs

pytestmark = pytest.mark.gpu


def load(text, catalog=None, **kw):
    from sparkalog_b200.datalog import ValueCatalog
    from sparkalog_b200.recursion import RelationStore

    catalog = catalog if catalog is not None else ValueCatalog()
    store = RelationStore()
    n = store.load_delimited(0, text, catalog, **kw)
    return store, catalog, n


def check(text, delimiter=",", has_header=False, catalog=None, want_catalog=None):
    store, cat, n = load(text, catalog, delimiter=delimiter, has_header=has_header)
    want_ids, want_cat = oracle.load_delimited(text, 2, delimiter, has_header, want_catalog)
    assert n == len(want_ids)
    f0, f1 = store.full(0)
    # A static relation keeps the file's rows in file order (duplicates too).
    got = list(zip(f0.tolist(), f1.tolist()))
    want = list(map(tuple, want_ids.tolist()))
    assert got == want
    by_id = sorted(want_cat.items(), key=lambda kv: kv[1])
    assert cat.values() == [v for v, _ in by_id]
    store.close()
    return cat, want_cat


def test_reference_vectors(cuda, known_answers):
    for case in known_answers["load_delimited"]:
        if "generated_rows" in case:
            text = "".join(case["format"].format(v=v) + "\n" for v in range(case["generated_rows"]))
        else:
            text = case["text"]
        check(text, case["delimiter"], case["has_header"])


def _random_text(rng, rows, distinct):
    pool = []
    for k in range(distinct):
        r = rng.integers(0, 4)
        if r == 0:
            pool.append(str(int(rng.integers(0, 1 << 32))))
        elif r == 1:
            pool.append(f"sym_{k}_é")
        elif r == 2:
            pool.append('"' + f'str {k} ""q"" ü' + '"')
        else:
            pool.append('"' + str(int(rng.integers(0, 1000))) + '"')  # a quoted number is a String
    lines = [f"{pool[rng.integers(0, distinct)]},{pool[rng.integers(0, distinct)]}" for _ in range(rows)]
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("rows,distinct,seed", [(50, 20, 1), (5_000, 800, 2), (200_000, 60_000, 3)])
def test_random_files_match_the_oracle(cuda, rows, distinct, seed):
    check(_random_text(np.random.default_rng(seed), rows, distinct))


def test_two_files_share_one_catalog(cuda):
    from sparkalog_b200.datalog import ValueCatalog

    rng = np.random.default_rng(4)
    a, b = _random_text(rng, 3_000, 500), _random_text(rng, 3_000, 700)
    cat = ValueCatalog()
    want = {}
    check(a, catalog=cat, want_catalog=want)
    check(b, catalog=cat, want_catalog=want)


def test_u32_entry_points_on_a_mixed_catalog(cuda):
    # intern_u32 continues the numbering; decode_u32 refuses a String's id.
    from sparkalog_b200.recursion import GenericExecutionError

    cat, want = check('7,"seven"\nx,7\n')
    ids = cat.intern(np.array([7, 8, 7, 9], dtype=np.uint32))
    assert ids.tolist() == [want[("u32", 7)], 3, want[("u32", 7)], 4]
    assert cat.decode(np.array([3, want[("u32", 7)]], dtype=np.uint32)).tolist() == [8, 7]
    with pytest.raises(GenericExecutionError):
        cat.decode(np.array([want[("string", "seven")]], dtype=np.uint32))


def test_errors(cuda):
    from sparkalog_b200.recursion import LoadError

    with pytest.raises(LoadError) as e:
        load('1,2\n"a",b,c\n')
    assert e.value.kind == "Arity" and e.value.line == 2
    for text in ['1,"open\n', '1,"a"b\n', "1,,2\n", "1,2,\n"]:
        with pytest.raises(oracle.OracleDelimitedError) as want:
            oracle.parse_delimited(text)
        with pytest.raises(LoadError) as got:
            load(text)
        assert (got.value.line, got.value.column) == (want.value.line, want.value.column)
