"""The no-allocation anti-join entry point agrees with the allocating one.

sparkalog_anti_join_u32_no_alloc serves callers that cannot allocate device
memory for the kernel's scratch (its scratch lives in a fixed array inside the
library). Here it is called through the C ABI and its outputs are compared,
bit for bit, with sparkalog_anti_join_u32 on the same inputs, for two calls in
a row: the second call must not see leftovers of the first, because both use
the same array. A third case fills the array exactly (the largest accepted
left side). After the calls, the entry point's own error word must read zero
through sparkalog_anti_join_u32_no_alloc_error. This file is named so that
pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

import oracle

MAX_ROWS = 1 << 27  # SPARKALOG_ANTI_JOIN_NO_ALLOC_MAX_LEFT_ROWS in include/sparkalog_b200.h


def _sorted_unique(rng, n, hi):
    a = rng.integers(0, hi, size=(n, 2)).astype(np.uint32)
    return oracle.distinct((a[:, 0], a[:, 1]))


def _run_both(torch, L, left, right):
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()
    lf, ls, rf, rs = dev(left[0]), dev(left[1]), dev(right[0]), dev(right[1])
    n = len(left[0])
    outputs = []
    for no_alloc in (False, True):
        flags = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        selected = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        count = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        o0 = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        o1 = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        if no_alloc:
            rc = L.sparkalog_anti_join_u32_no_alloc(lf.data_ptr(), ls.data_ptr(), n, rf.data_ptr(), rs.data_ptr(),
                                                    len(right[0]), flags.data_ptr(), selected.data_ptr(),
                                                    count.data_ptr(), o0.data_ptr(), o1.data_ptr(), None)
        else:
            size = ctypes.c_size_t(0)
            assert L.sparkalog_anti_join_u32_temporary_bytes(flags.data_ptr(), selected.data_ptr(), count.data_ptr(),
                                                             n, ctypes.byref(size), None) == 0
            temp = torch.empty(max(size.value, 1), dtype=torch.uint8, device="cuda")
            rc = L.sparkalog_anti_join_u32(lf.data_ptr(), ls.data_ptr(), n, rf.data_ptr(), rs.data_ptr(),
                                           len(right[0]), flags.data_ptr(), selected.data_ptr(), count.data_ptr(),
                                           o0.data_ptr(), o1.data_ptr(), temp.data_ptr(), size.value, None)
        assert rc == 0
        torch.cuda.synchronize()
        k = int(count.item())
        outputs.append((k, flags.cpu().numpy(), selected[:k].cpu().numpy(), o0[:k].cpu().numpy(),
                        o1[:k].cpu().numpy()))
    return outputs


@pytest.mark.gpu
def test_no_alloc_anti_join_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("GPU test without a CUDA device")
    from sparkalog_b200 import _native

    L = _native.load()
    rng = np.random.default_rng(2027)
    # First call: many tiles; second call: fewer rows, so stale scratch from
    # the first call would be visible if it were not cleared.
    cases = [(_sorted_unique(rng, 900_000, 2_000), _sorted_unique(rng, 700_000, 2_000)),
             (_sorted_unique(rng, 5_000, 300), _sorted_unique(rng, 20_000, 300))]
    for left, right in cases:
        alloc, no_alloc = _run_both(torch, L, left, right)
        assert alloc[0] == no_alloc[0]
        for a, b in zip(alloc[1:], no_alloc[1:]):
            assert np.array_equal(a, b)
        want = oracle.anti_join(left, right)
        assert np.array_equal(no_alloc[3].view(np.uint32), want[0])
        assert np.array_equal(no_alloc[4].view(np.uint32), want[1])
    bits = ctypes.c_uint32(0xFFFFFFFF)
    assert L.sparkalog_anti_join_u32_no_alloc_error(ctypes.byref(bits), 1) == 0
    assert bits.value == 0
    assert L.sparkalog_anti_join_u32_no_alloc_error(ctypes.byref(bits), 0) == 0
    assert bits.value == 0


@pytest.mark.gpu
def test_no_alloc_anti_join_at_its_maximum_left_rows():
    """Exactly SPARKALOG_ANTI_JOIN_NO_ALLOC_MAX_LEFT_ROWS left rows: the call
    clears every status word of the array. The left side is generated on the
    device (sorted and unique by construction: first = i >> 4, second =
    3 * (i & 15)); the right side removes every row whose first column is a
    multiple of 1,000, so the expected output is known in closed form."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("GPU test without a CUDA device")
    from sparkalog_b200 import _native

    L = _native.load()
    n = MAX_ROWS
    i = torch.arange(n, dtype=torch.int64, device="cuda")
    lf = (i >> 4).to(torch.int32)
    ls = ((i & 15) * 3).to(torch.int32)
    del i
    keys = torch.arange(0, n >> 4, 1000, dtype=torch.int64, device="cuda")
    rf = keys.repeat_interleave(16).to(torch.int32)
    rs = (torch.arange(16, dtype=torch.int64, device="cuda") * 3).repeat(len(keys)).to(torch.int32)
    del keys
    results = []
    for no_alloc in (False, True):
        flags = torch.empty(n, dtype=torch.int32, device="cuda")
        selected = torch.empty(n, dtype=torch.int32, device="cuda")
        count = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        o0 = torch.empty(n, dtype=torch.int32, device="cuda")
        o1 = torch.empty(n, dtype=torch.int32, device="cuda")
        if no_alloc:
            rc = L.sparkalog_anti_join_u32_no_alloc(lf.data_ptr(), ls.data_ptr(), n, rf.data_ptr(), rs.data_ptr(),
                                                    len(rf), flags.data_ptr(), selected.data_ptr(), count.data_ptr(),
                                                    o0.data_ptr(), o1.data_ptr(), None)
        else:
            size = ctypes.c_size_t(0)
            assert L.sparkalog_anti_join_u32_temporary_bytes(flags.data_ptr(), selected.data_ptr(), count.data_ptr(),
                                                             n, ctypes.byref(size), None) == 0
            temp = torch.empty(max(size.value, 1), dtype=torch.uint8, device="cuda")
            rc = L.sparkalog_anti_join_u32(lf.data_ptr(), ls.data_ptr(), n, rf.data_ptr(), rs.data_ptr(), len(rf),
                                           flags.data_ptr(), selected.data_ptr(), count.data_ptr(), o0.data_ptr(),
                                           o1.data_ptr(), temp.data_ptr(), size.value, None)
        assert rc == 0
        torch.cuda.synchronize()
        k = int(count.item())
        results.append((k, o0[:k].clone(), o1[:k].clone()))
        del flags, selected, o0, o1
    (ka, a0, a1), (kb, b0, b1) = results
    assert ka == kb == n - len(rf)
    assert torch.equal(a0, b0) and torch.equal(a1, b1)
    assert not bool(((b0 % 1000) == 0).any())
    bits = ctypes.c_uint32(0xFFFFFFFF)
    assert L.sparkalog_anti_join_u32_no_alloc_error(ctypes.byref(bits), 1) == 0
    assert bits.value == 0


def test_no_alloc_anti_join_rejects_rows_beyond_its_maximum():
    # The size check comes before any device work, so this needs no GPU.
    from sparkalog_b200 import _native

    L = _native.load()
    dummy = 256  # never dereferenced: the call is rejected first
    rc = L.sparkalog_anti_join_u32_no_alloc(dummy, dummy, MAX_ROWS + 1, dummy, dummy, 1, dummy, dummy, dummy, dummy,
                                            dummy, None)
    assert rc == 1  # cudaErrorInvalidValue
    assert L.sparkalog_anti_join_u32_no_alloc(dummy, dummy, 1, dummy, dummy, 1, dummy, dummy, None, dummy, dummy,
                                              None) == 1


def test_no_alloc_error_getter_is_exported_and_checks_its_argument():
    # A null output is rejected before any device work, so this needs no GPU.
    from sparkalog_b200 import _native

    L = _native.load()
    assert L.sparkalog_anti_join_u32_no_alloc_error(None, 1) == 1  # cudaErrorInvalidValue
