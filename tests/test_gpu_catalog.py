"""GPU value interning (ValueCatalog, crates/sparkalog-datalog/src/catalog.rs:98-127) against the
oracle's one-value-at-a-time restatement: ids bit-exact across batches, decode round trips."""

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_interning_matches_first_appearance(cuda):
    from sparkalog_b200.datalog import ValueCatalog

    torch = cuda
    rng = np.random.default_rng(3)
    cat = ValueCatalog()
    ref = {}
    batches = [np.array([], dtype=np.uint32), np.array([7, 3, 7, 0xFFFFFFFF, 3, 0], dtype=np.uint32),
               rng.integers(0, 1000, size=5000).astype(np.uint32),
               rng.integers(0, 1 << 32, size=300_000, dtype=np.uint64).astype(np.uint32),
               rng.integers(0, 50_000, size=1_000_000).astype(np.uint32)]
    for i, batch in enumerate(batches):
        want, ref = oracle.intern(batch, ref)
        got = cat.intern(batch) if i % 2 == 0 else cat.intern(torch.from_numpy(batch.view(np.int32)).cuda())
        got = got if isinstance(got, np.ndarray) else got.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want)
        assert len(cat) == len(ref)
    ids = np.arange(len(ref), dtype=np.uint32)
    inverse = np.empty(len(ref), dtype=np.uint32)
    for v, k in ref.items():
        inverse[k] = v
    assert np.array_equal(cat.decode(ids), inverse)
    from sparkalog_b200.recursion import GenericExecutionError

    with pytest.raises(GenericExecutionError):
        cat.decode(np.array([len(ref)], dtype=np.uint32))


def test_interning_rows_in_insert_order(cuda):
    # Database::insert interns row[0] then row[1] of each row in turn.
    from sparkalog_b200.datalog import ValueCatalog

    first = np.array([10, 30, 20, 10], dtype=np.uint32)
    second = np.array([20, 10, 40, 30], dtype=np.uint32)
    cat = ValueCatalog()
    f, s = cat.intern_rows(first, second)
    want, _ = oracle.intern(np.stack([first, second], axis=1).reshape(-1))
    assert f.tolist() == want[0::2].tolist() and s.tolist() == want[1::2].tolist()
    assert f.tolist() == [0, 2, 1, 0] and s.tolist() == [1, 0, 3, 2]
