"""GPU parity of the reference-compatible operator ABI (Tier A) against the oracle.

Mirrors the reference's cross-backend equivalence tests
(crates/sparkalog-execution/src/lib.rs:2031-2651): every CUDA output column
equals the serial CPU output. All comparisons are bit-exact (integer work).
When the reference's own column_ops.cu has been built for sm_100a
(oracle/_ref), its outputs are compared too.
"""

import ctypes

import numpy as np
import pytest

import oracle
from conftest import cols, pairs

pytestmark = pytest.mark.gpu


def ex():
    from sparkalog_b200 import execution

    return execution


def rel(columns):
    return ex().Relation.from_host(*columns)


def out_pairs(workspace):
    return pairs(workspace.output.to_host())


def test_known_answers_all_operators(cuda, known_answers):
    E = ex()
    from sparkalog_b200.relational import (BinaryDistinct, BinaryEqualityJoin, JoinInput, JoinProjection,
                                           SortedBinaryAntiJoin, SortedBinaryUnion)

    stream = E.CudaStream()
    for case in known_answers["distinct"]:
        ws = E.DistinctWorkspace()
        E.distinct_cuda(rel(cols(case["input"])), BinaryDistinct(), ws, stream)
        assert out_pairs(ws) == case["expected"], case["source"]
    for case in known_answers["anti_join"]:
        ws = E.AntiJoinWorkspace()
        E.anti_join_cuda(rel(cols(case["left"])), rel(cols(case["right"])), SortedBinaryAntiJoin(), ws, stream)
        assert out_pairs(ws) == case["expected"], case["source"]
    for case in known_answers["union"]:
        ws = E.UnionWorkspace()
        E.union_cuda(rel(cols(case["left"])), rel(cols(case["right"])), SortedBinaryUnion(), ws, stream)
        assert out_pairs(ws) == case["expected"], case["source"]
    for case in known_answers["join"]:
        left, right = rel(cols(case["left"])), rel(cols(case["right"]))
        index = E.U32RangeIndex.build(right, case["right_key"])
        plan = BinaryEqualityJoin(case["left_key"], case["right_key"],
                                  tuple(JoinProjection(JoinInput(s), c) for s, c in case["projection"]))
        ws = E.JoinWorkspace()
        E.join_cuda(left, right, index, plan, ws, stream)
        assert out_pairs(ws) == case["expected"], case["source"]


def random_sorted_unique(rng, n, hi):
    a = rng.integers(0, hi, size=(n, 2)).astype(np.uint32)
    return oracle.distinct((a[:, 0], a[:, 1]))


@pytest.mark.parametrize("n", [1, 2, 255, 4096, 4097, 100_000, 1_000_003])
def test_distinct_random(cuda, n):
    E = ex()
    from sparkalog_b200.relational import BinaryDistinct

    rng = np.random.default_rng(n)
    hi = max(4, int(np.sqrt(n)))
    a = rng.integers(0, hi, size=(n, 2)).astype(np.uint32)
    if n > 10:
        a[::7, 0] = 0xFFFFFFFF  # exercise the top digits
    ws = E.DistinctWorkspace()
    E.distinct_cuda(rel((a[:, 0], a[:, 1])), BinaryDistinct(), ws, E.CudaStream())
    want = oracle.distinct((a[:, 0], a[:, 1]))
    got = ws.output.to_host()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_distinct_full_64_bit_keys(cuda):
    E = ex()
    from sparkalog_b200.relational import BinaryDistinct

    rng = np.random.default_rng(99)
    a = rng.integers(0, 1 << 32, size=(300_000, 2), dtype=np.uint64).astype(np.uint32)
    a = np.concatenate([a, a[:50_000]])
    ws = E.DistinctWorkspace()
    E.distinct_cuda(rel((a[:, 0], a[:, 1])), BinaryDistinct(), ws, E.CudaStream())
    want = oracle.distinct((a[:, 0], a[:, 1]))
    got = ws.output.to_host()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


@pytest.mark.parametrize("nl,nr,hi", [(1, 0, 10), (0, 5, 10), (5000, 3, 50), (3, 5000, 50), (200_000, 150_000, 700),
                                      (50_000, 3_000_000, 3000), (1_000_000, 1_000, 5000)])
def test_anti_join_and_union_random(cuda, nl, nr, hi):
    E = ex()
    from sparkalog_b200.relational import SortedBinaryAntiJoin, SortedBinaryUnion

    rng = np.random.default_rng(nl * 7 + nr)
    left = random_sorted_unique(rng, nl, hi)
    right = random_sorted_unique(rng, nr, hi)
    stream = E.CudaStream()
    ws = E.AntiJoinWorkspace()
    E.anti_join_cuda(rel(left), rel(right), SortedBinaryAntiJoin(), ws, stream)
    want = oracle.anti_join(left, right)
    got = ws.output.to_host()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    # flags / selected keep the reference's meaning.
    n = len(left[0])
    if n:
        flags = ws.flags[:n].cpu().numpy().view(np.uint32)
        sel = ws.selected[: len(want[0])].cpu().numpy().view(np.uint32)
        assert np.array_equal(np.nonzero(flags)[0].astype(np.uint32), sel)
    wu = E.UnionWorkspace()
    E.union_cuda(rel(left), rel(right), SortedBinaryUnion(), wu, stream)
    want_u = oracle.union(left, right)
    got_u = wu.output.to_host()
    assert np.array_equal(got_u[0], want_u[0]) and np.array_equal(got_u[1], want_u[1])


def test_union_with_duplicates_inside_inputs(cuda):
    E = ex()
    from sparkalog_b200.relational import SortedBinaryUnion

    rng = np.random.default_rng(3)
    a = np.sort(rng.integers(0, 1 << 20, size=400_000).astype(np.uint64))
    b = np.sort(rng.integers(0, 1 << 20, size=300_000).astype(np.uint64))
    left = ((a >> np.uint64(10)).astype(np.uint32), (a & np.uint64(1023)).astype(np.uint32))
    right = ((b >> np.uint64(10)).astype(np.uint32), (b & np.uint64(1023)).astype(np.uint32))
    ws = E.UnionWorkspace()
    E.union_cuda(rel(left), rel(right), SortedBinaryUnion(), ws, E.CudaStream())
    want = oracle.union(left, right)
    got = ws.output.to_host()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_anti_join_unsorted_left_matches_reference_semantics(cuda):
    # The reference's CUDA anti-join checks each left row independently
    # (binary search per row), so an unsorted left input still yields, in
    # left order, the rows absent from the sorted right input.
    E = ex()
    from sparkalog_b200.relational import SortedBinaryAntiJoin

    rng = np.random.default_rng(17)
    right = random_sorted_unique(rng, 50_000, 400)
    raw = rng.integers(0, 400, size=(60_000, 2)).astype(np.uint32)
    ws = E.AntiJoinWorkspace()
    E.anti_join_cuda(rel((raw[:, 0], raw[:, 1])), rel(right), SortedBinaryAntiJoin(), ws, E.CudaStream())
    rset = set(zip(right[0].tolist(), right[1].tolist()))
    want = [[int(x), int(y)] for x, y in raw if (int(x), int(y)) not in rset]
    assert out_pairs(ws) == want


@pytest.mark.parametrize("nl,ne,hub", [(10, 40, False), (5000, 20_000, False), (300_000, 1_000_000, False),
                                       (20_000, 50_000, True)])
def test_join_random(cuda, nl, ne, hub):
    E = ex()
    from sparkalog_b200.relational import path_join

    rng = np.random.default_rng(nl + ne)
    nodes = max(16, ne // 2)
    edges = rng.integers(0, nodes, size=(ne, 2)).astype(np.uint32)
    if hub:
        edges[: ne // 3, 0] = 7  # one key with many matches
    edges = oracle.btree_pairs(edges[:, 0], edges[:, 1])
    left = rng.integers(0, nodes, size=(nl, 2)).astype(np.uint32)
    left = (left[:, 0], left[:, 1])
    if hub:
        left[1][::5] = 7
    right = rel(edges)
    index = E.U32RangeIndex.build(right, 0)
    ws = E.JoinWorkspace()
    E.join_cuda(rel(left), right, index, path_join(), ws, E.CudaStream())
    want = oracle.join(left, edges)
    got = ws.output.to_host()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    # counts/offsets keep the reference's meaning.
    n = len(left[0])
    counts = ws.counts[:n].cpu().numpy().view(np.uint64)
    offsets = ws.offsets[:n].cpu().numpy().view(np.uint64)
    assert int(counts.sum()) == len(want[0])
    assert np.array_equal(offsets, np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint64))


def test_empty_inputs_and_null_checks(cuda):
    E = ex()
    from sparkalog_b200 import _native
    from sparkalog_b200.relational import BinaryDistinct, SortedBinaryAntiJoin, SortedBinaryUnion

    stream = E.CudaStream()
    empty = rel(cols([]))
    ws = E.DistinctWorkspace()
    E.distinct_cuda(empty, BinaryDistinct(), ws, stream)
    assert len(ws.output) == 0
    wa = E.AntiJoinWorkspace()
    E.anti_join_cuda(empty, rel(cols([[1, 2]])), SortedBinaryAntiJoin(), wa, stream)
    assert len(wa.output) == 0
    wu = E.UnionWorkspace()
    E.union_cuda(empty, empty, SortedBinaryUnion(), wu, stream)
    assert len(wu.output) == 0
    L = _native.load()
    # A null required pointer is cudaErrorInvalidValue (1), as in column_ops.cu.
    size = ctypes.c_size_t(0)
    assert L.sparkalog_distinct_u32_temporary_bytes(None, None, None, 5, ctypes.byref(size), None) == 1
    assert L.sparkalog_union_u32(None, None, 0, None, None, 0, None, None, None, None, None, None, None, None, 0,
                                 None) == 1
    assert L.sparkalog_anti_join_u32(None, None, 3, None, None, 0, None, None, None, None, None, None, 0, None) == 1


def _ref_call_distinct(ref, first, second, torch):
    n = len(first)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()
    f, s = d(first), d(second)
    packed = torch.empty(max(n, 1), dtype=torch.int64, device="cuda")
    scratch = torch.empty_like(packed)
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    o0 = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    o1 = torch.empty_like(o0)
    tb = ctypes.c_size_t(0)
    vp = ctypes.c_void_p
    ref.sparkalog_distinct_u32_temporary_bytes.argtypes = [vp, vp, vp, ctypes.c_size_t,
                                                           ctypes.POINTER(ctypes.c_size_t), vp]
    ref.sparkalog_distinct_u32.argtypes = [vp, vp, ctypes.c_size_t, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
    assert ref.sparkalog_distinct_u32_temporary_bytes(packed.data_ptr(), scratch.data_ptr(), count.data_ptr(), n,
                                                      ctypes.byref(tb), None) == 0
    tmp = torch.empty(max(tb.value, 1), dtype=torch.uint8, device="cuda")
    assert ref.sparkalog_distinct_u32(f.data_ptr(), s.data_ptr(), n, packed.data_ptr(), scratch.data_ptr(),
                                      count.data_ptr(), o0.data_ptr(), o1.data_ptr(), tmp.data_ptr(), tb.value,
                                      None) == 0
    torch.cuda.synchronize()
    u = int(count.item())
    return o0[:u].cpu().numpy().view(np.uint32), o1[:u].cpu().numpy().view(np.uint32)


def test_against_reference_cuda_build(cuda):
    """The reference's own column_ops.cu (built for sm_100a from its source) agrees."""
    ref = oracle.reference_cuda()
    if ref is None:
        pytest.skip("reference CUDA library not built (oracle/_ref)")
    E = ex()
    from sparkalog_b200.relational import BinaryDistinct

    rng = np.random.default_rng(1234)
    a = rng.integers(0, 5000, size=(500_000, 2)).astype(np.uint32)
    r0, r1 = _ref_call_distinct(ref, a[:, 0], a[:, 1], cuda)
    ws = E.DistinctWorkspace()
    E.distinct_cuda(rel((a[:, 0], a[:, 1])), BinaryDistinct(), ws, E.CudaStream())
    g0, g1 = ws.output.to_host()
    assert np.array_equal(r0, g0) and np.array_equal(r1, g1)


def test_device_error_bits_clear(cuda):
    from sparkalog_b200 import _native

    bits = ctypes.c_uint32(123)
    assert _native.load().sparkalog_b200_device_error(ctypes.byref(bits), 1) == 0
    assert bits.value == 0


def test_filter_known_answers_and_oracle(cuda, known_answers):
    # lib.rs:2015-2027, 2403-2445 plus random columns against the oracle.
    E = ex()
    from sparkalog_b200.relational import U32Predicate

    torch = cuda
    stream = E.CudaStream()
    ws = E.FilterWorkspace()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()
    for case in known_answers["filter"]:
        if "values_mod" in case:
            n, m = case["values_mod"]
            values = np.arange(n, dtype=np.uint32) % m
            E.filter_cuda(dev(values), U32Predicate(case["op"]), case["operand"], ws, stream)
            assert ws.selected == case["expected_count"]
            assert np.array_equal(ws.selection_host(), oracle.filter_serial(values, case["op"], case["operand"]))
            continue
        for op, operand, want in case["cases"]:
            E.filter_cuda(dev(case["values"]), U32Predicate(op), operand, ws, stream)
            assert ws.selection_host().tolist() == want, case["source"]
    rng = np.random.default_rng(77)
    for n in (1, 2047, 2048, 2049, 1_000_003):
        values = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
        values[::7] = 12345
        for op in range(6):
            operand = 12345 if op in (0, 1) else int(values[n // 2])
            E.filter_cuda(dev(values), U32Predicate(op), operand, ws, stream)
            assert np.array_equal(ws.selection_host(), oracle.filter_parallel(values, op, operand))
            flags = ws.flags[:n].cpu().numpy().view(np.uint32)
            want = np.zeros(n, dtype=np.uint32)
            want[oracle.filter_parallel(values, op, operand)] = 1
            assert np.array_equal(flags, want)


def test_filter_fill_add_one_edges(cuda, known_answers):
    from sparkalog_b200 import _native

    E = ex()
    torch = cuda
    stream = E.CudaStream()
    L = _native.load()
    size = ctypes.c_size_t(0)
    # Null checks and empty inputs as in column_ops.cu:252-336.
    assert L.sparkalog_filter_u32_temporary_bytes(None, None, None, 0, ctypes.byref(size), None) == 1
    assert L.sparkalog_filter_u32(None, 0, 0, 0, None, None, None, None, 0, None) == 1
    assert L.sparkalog_fill_mod_u32(None, 0, 0, None) == 1
    assert L.sparkalog_fill_mod_u32(None, 0, 5, None) == 0
    assert L.sparkalog_add_one_i32(None, 3, None) == 1
    count = torch.full((1,), 99, dtype=torch.int32, device="cuda")
    assert L.sparkalog_filter_u32(None, 0, 0, 0, None, None, count.data_ptr(), None, 0, stream.raw) == 0
    stream.synchronize()
    assert int(count.item()) == 0
    # fill_mod: lib.rs:2448-2459.
    fm = known_answers["fill_mod"]
    col = torch.zeros(fm["len"], dtype=torch.int32, device="cuda")
    E.fill_mod_u32(col, fm["modulus"], stream)
    stream.synchronize()
    assert col.cpu().numpy().tolist() == [i % fm["modulus"] for i in range(fm["len"])]
    E.add_one_i32(col, stream)
    stream.synchronize()
    assert col.cpu().numpy().tolist() == [i % fm["modulus"] + 1 for i in range(fm["len"])]


def test_filter_against_reference_cuda_build(cuda):
    """The reference's own sparkalog_filter_u32 (column_ops.cu built for sm_100a) agrees."""
    ref = oracle.reference_cuda()
    if ref is None:
        pytest.skip("reference CUDA library not built (oracle/_ref)")
    E = ex()
    from sparkalog_b200.relational import U32Predicate

    torch = cuda
    vp = ctypes.c_void_p
    ref.sparkalog_filter_u32_temporary_bytes.argtypes = [vp, vp, vp, ctypes.c_size_t,
                                                         ctypes.POINTER(ctypes.c_size_t), vp]
    ref.sparkalog_filter_u32.argtypes = [vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp, vp,
                                         ctypes.c_size_t, vp]
    rng = np.random.default_rng(5)
    n = 300_000
    values = rng.integers(0, 1000, size=n).astype(np.uint32)
    col = torch.from_numpy(values.view(np.int32)).cuda()
    flags = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.zeros(n, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    tb = ctypes.c_size_t(0)
    assert ref.sparkalog_filter_u32_temporary_bytes(flags.data_ptr(), out.data_ptr(), count.data_ptr(), n,
                                                    ctypes.byref(tb), None) == 0
    tmp = torch.empty(max(tb.value, 1), dtype=torch.uint8, device="cuda")
    ws = E.FilterWorkspace()
    stream = E.CudaStream()
    for op in range(6):
        assert ref.sparkalog_filter_u32(col.data_ptr(), n, op, 500, flags.data_ptr(), out.data_ptr(),
                                        count.data_ptr(), tmp.data_ptr(), tb.value, None) == 0
        torch.cuda.synchronize()
        want = out[:int(count.item())].cpu().numpy().view(np.uint32)
        E.filter_cuda(col, U32Predicate(op), 500, ws, stream)
        assert np.array_equal(ws.selection_host(), want)
