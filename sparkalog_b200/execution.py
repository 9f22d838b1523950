"""Physical operators through the reference-compatible C ABI (Tier A).

Mirrors the CUDA half of crates/sparkalog-execution/src/lib.rs: ``CudaStream``
(:241-277), ``distinct_cuda`` (:465-531), ``anti_join_cuda`` (:814-886),
``union_cuda`` (:1098-1177) and ``join_cuda`` (:1549-1648), with the same
workspace-based calling pattern and the same error conditions. Relations are
pairs of device columns (``torch`` uint32 storage viewed as int32); PyTorch is
used only to hold device memory and streams.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .relational import (BinaryDistinct, BinaryEqualityJoin, JoinInput, SortedBinaryAntiJoin, SortedBinaryUnion,
                         U32Predicate)

U32_MAX = 0xFFFFFFFF


class CudaError(RuntimeError):
    """execution::Error::Cuda { operation, code } (lib.rs:171-239)."""

    def __init__(self, operation: str, code: int):
        super().__init__(f"{operation} failed with CUDA error {code}")
        self.operation = operation
        self.code = code


class TooManyRows(ValueError):
    """execution::Error::TooManyRows (lib.rs:325-331)."""


class MissingColumn(ValueError):
    """execution::Error::MissingColumn."""


class IndexSourceMismatch(ValueError):
    """execution::Error::IndexSourceMismatch."""


def _check(operation: str, code: int) -> None:
    if code != 0:
        raise CudaError(operation, code)


def check_row_count(rows: int) -> None:
    if rows > U32_MAX:
        raise TooManyRows(f"{rows} rows cannot be represented by u32 row IDs")


class CudaStream:
    """A non-blocking CUDA stream (lib.rs:241-277)."""

    def __init__(self, device: int | None = None):
        self.torch_stream = torch.cuda.Stream(device=device)

    @property
    def raw(self) -> int:
        return self.torch_stream.cuda_stream

    def synchronize(self) -> None:
        _check("cudaStreamSynchronize", _native.load().sparkalog_stream_synchronize(self.raw))


def _dev_u32(n: int) -> torch.Tensor:
    return torch.empty(max(n, 1), dtype=torch.int32, device="cuda")


def _dev_u64(n: int) -> torch.Tensor:
    return torch.empty(max(n, 1), dtype=torch.int64, device="cuda")


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


class Relation:
    """A binary relation as two device u32 columns (storage Relation, storage/src/lib.rs:157-210)."""

    def __init__(self, first: torch.Tensor, second: torch.Tensor, rows: int):
        self.columns = [first, second]
        self.rows = rows

    @classmethod
    def from_host(cls, first, second) -> "Relation":
        a = np.ascontiguousarray(np.asarray(first, dtype=np.uint32)).view(np.int32)
        b = np.ascontiguousarray(np.asarray(second, dtype=np.uint32)).view(np.int32)
        n = len(a)
        c0 = _dev_u32(n)
        c1 = _dev_u32(n)
        if n:
            c0[:n].copy_(torch.from_numpy(a))
            c1[:n].copy_(torch.from_numpy(b))
        return cls(c0, c1, n)

    @classmethod
    def from_pairs(cls, pairs) -> "Relation":
        arr = np.asarray(pairs, dtype=np.uint32).reshape(-1, 2)
        return cls.from_host(arr[:, 0], arr[:, 1])

    def __len__(self) -> int:
        return self.rows

    def column(self, index: int) -> torch.Tensor:
        if index not in (0, 1):
            raise MissingColumn(f"relation has no column {index}")
        return self.columns[index]

    def to_host(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.rows
        return (self.columns[0][:n].cpu().numpy().view(np.uint32).copy(),
                self.columns[1][:n].cpu().numpy().view(np.uint32).copy())


class U32RangeIndex:
    """Sparse sorted range index (storage/src/lib.rs:345-423), built on the host as in the
    reference (U32RangeIndex::build_slice, :357-393) and held on the device."""

    def __init__(self, values: np.ndarray):
        v = np.asarray(values, dtype=np.uint32)
        n = len(v)
        check_row_count(n)
        rows = np.lexsort((np.arange(n, dtype=np.uint32), v)).astype(np.uint32)
        sorted_vals = v[rows]
        if n:
            change = np.ones(n, dtype=bool)
            change[1:] = sorted_vals[1:] != sorted_vals[:-1]
            keys = sorted_vals[change]
            starts = np.concatenate([np.nonzero(change)[0], [n]]).astype(np.uint32)
        else:
            keys = np.zeros(0, dtype=np.uint32)
            starts = np.zeros(1, dtype=np.uint32)
        self.source_rows = n
        self.host_keys, self.host_starts, self.host_rows = keys, starts, rows
        self.keys = Relation.from_host(keys, keys).columns[0]
        self.starts = Relation.from_host(starts, starts).columns[0]
        self.rows = Relation.from_host(rows, rows).columns[0]
        self.unique_keys = len(keys)

    @classmethod
    def build(cls, relation: Relation, column: int) -> "U32RangeIndex":
        first, second = relation.to_host()
        return cls(first if column == 0 else second)


@dataclass
class _Temp:
    buf: torch.Tensor | None = None

    def reserve(self, nbytes: int) -> torch.Tensor:
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device="cuda")
        return self.buf


class JoinWorkspace:
    """Counts, offsets, total and output of a join (storage/src/lib.rs:497-595)."""

    def __init__(self):
        self.output = Relation(_dev_u32(0), _dev_u32(0), 0)
        self.counts = _dev_u64(0)
        self.offsets = _dev_u64(0)
        self.total = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.temp = _Temp()


class DistinctWorkspace:
    """Packed/scratch sort buffers, count and output (storage/src/lib.rs:598-685)."""

    def __init__(self):
        self.output = Relation(_dev_u32(0), _dev_u32(0), 0)
        self.packed = _dev_u64(0)
        self.scratch = _dev_u64(0)
        self.count = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.temp = _Temp()


class AntiJoinWorkspace:
    """Flags, selection, count and output (storage/src/lib.rs:688-769)."""

    def __init__(self):
        self.output = Relation(_dev_u32(0), _dev_u32(0), 0)
        self.flags = _dev_u32(0)
        self.selected = _dev_u32(0)
        self.count = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.temp = _Temp()


class UnionWorkspace:
    """Packed inputs, merged/unique scratch, count and output (storage/src/lib.rs:772-870)."""

    def __init__(self):
        self.output = Relation(_dev_u32(0), _dev_u32(0), 0)
        self.left = _dev_u64(0)
        self.right = _dev_u64(0)
        self.merged = _dev_u64(0)
        self.unique = _dev_u64(0)
        self.count = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.temp = _Temp()


class FilterWorkspace:
    """Flags, selection (row ids) and count of a filter (storage/src/lib.rs:499-595)."""

    def __init__(self):
        self.flags = _dev_u32(0)
        self.selection = _dev_u32(0)
        self.count = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.selected = 0
        self.temp = _Temp()

    def selection_host(self) -> np.ndarray:
        return self.selection[:self.selected].cpu().numpy().view(np.uint32)


def _grow_u32(t: torch.Tensor, n: int) -> torch.Tensor:
    return t if t.numel() >= max(n, 1) else _dev_u32(n)


def _grow_u64(t: torch.Tensor, n: int) -> torch.Tensor:
    return t if t.numel() >= max(n, 1) else _dev_u64(n)


def _read_count(t: torch.Tensor, stream: CudaStream) -> int:
    stream.synchronize()
    v = int(t[0].item())
    return v & (U32_MAX if t.dtype == torch.int32 else 0xFFFFFFFFFFFFFFFF)


def filter_cuda(column: torch.Tensor, predicate: U32Predicate, operand: int, workspace: FilterWorkspace,
                stream: CudaStream) -> None:
    """Ascending row ids whose value satisfies the predicate (filter_cuda, lib.rs:1809-1875, plus its wait)."""
    L = _native.load()
    n = int(column.numel())
    check_row_count(n)
    ws = workspace
    ws.flags = _grow_u32(ws.flags, n)
    ws.selection = _grow_u32(ws.selection, n)
    temp_bytes = ctypes.c_size_t(0)
    _check("sparkalog_filter_u32_temporary_bytes",
           L.sparkalog_filter_u32_temporary_bytes(_ptr(ws.flags), _ptr(ws.selection), _ptr(ws.count), n,
                                                  ctypes.byref(temp_bytes), stream.raw))
    temp = ws.temp.reserve(temp_bytes.value)
    _check("sparkalog_filter_u32",
           L.sparkalog_filter_u32(_ptr(column), n, int(predicate), int(operand) & U32_MAX, _ptr(ws.flags),
                                  _ptr(ws.selection), _ptr(ws.count), _ptr(temp), temp_bytes.value, stream.raw))
    ws.selected = _read_count(ws.count, stream)


def fill_mod_u32(column: torch.Tensor, modulus: int, stream: CudaStream) -> None:
    """column[i] = i % modulus (fill_mod_u32, lib.rs:1926-1950)."""
    _check("sparkalog_fill_mod_u32", _native.load().sparkalog_fill_mod_u32(_ptr(column), int(column.numel()),
                                                                            int(modulus), stream.raw))


def add_one_i32(column: torch.Tensor, stream: CudaStream) -> None:
    """column[i] += 1 (add_one_i32, lib.rs:305-320)."""
    _check("sparkalog_add_one_i32", _native.load().sparkalog_add_one_i32(_ptr(column), int(column.numel()),
                                                                          stream.raw))


def distinct_cuda(input: Relation, plan: BinaryDistinct, workspace: DistinctWorkspace, stream: CudaStream) -> None:
    """Sort and deduplicate binary tuples (distinct_cuda, lib.rs:465-531, plus PendingDistinct::wait)."""
    L = _native.load()
    check_row_count(len(input))
    first, second = input.column(plan.columns[0]), input.column(plan.columns[1])
    n = len(input)
    ws = workspace
    ws.packed = _grow_u64(ws.packed, n)
    ws.scratch = _grow_u64(ws.scratch, n)
    out0 = _grow_u32(ws.output.columns[0], n)
    out1 = _grow_u32(ws.output.columns[1], n)
    ws.output = Relation(out0, out1, 0)
    temp_bytes = ctypes.c_size_t(0)
    _check("sparkalog_distinct_u32_temporary_bytes",
           L.sparkalog_distinct_u32_temporary_bytes(_ptr(ws.packed), _ptr(ws.scratch), _ptr(ws.count), n,
                                                    ctypes.byref(temp_bytes), stream.raw))
    temp = ws.temp.reserve(temp_bytes.value)
    _check("sparkalog_distinct_u32",
           L.sparkalog_distinct_u32(_ptr(first), _ptr(second), n, _ptr(ws.packed), _ptr(ws.scratch), _ptr(ws.count),
                                    _ptr(out0), _ptr(out1), _ptr(temp), temp_bytes.value, stream.raw))
    ws.output.rows = _read_count(ws.count, stream)


def anti_join_cuda(left: Relation, right: Relation, plan: SortedBinaryAntiJoin, workspace: AntiJoinWorkspace,
                   stream: CudaStream) -> None:
    """Stable sorted anti-join (anti_join_cuda, lib.rs:814-886, plus PendingAntiJoin::wait)."""
    L = _native.load()
    check_row_count(len(left))
    check_row_count(len(right))
    lf, ls = left.column(plan.left[0]), left.column(plan.left[1])
    rf, rs = right.column(plan.right[0]), right.column(plan.right[1])
    n = len(left)
    ws = workspace
    ws.flags = _grow_u32(ws.flags, n)
    ws.selected = _grow_u32(ws.selected, n)
    out0 = _grow_u32(ws.output.columns[0], n)
    out1 = _grow_u32(ws.output.columns[1], n)
    ws.output = Relation(out0, out1, 0)
    temp_bytes = ctypes.c_size_t(0)
    _check("sparkalog_anti_join_u32_temporary_bytes",
           L.sparkalog_anti_join_u32_temporary_bytes(_ptr(ws.flags), _ptr(ws.selected), _ptr(ws.count), n,
                                                     ctypes.byref(temp_bytes), stream.raw))
    temp = ws.temp.reserve(temp_bytes.value)
    _check("sparkalog_anti_join_u32",
           L.sparkalog_anti_join_u32(_ptr(lf), _ptr(ls), n, _ptr(rf), _ptr(rs), len(right), _ptr(ws.flags),
                                     _ptr(ws.selected), _ptr(ws.count), _ptr(out0), _ptr(out1), _ptr(temp),
                                     temp_bytes.value, stream.raw))
    ws.output.rows = _read_count(ws.count, stream)


def union_cuda(left: Relation, right: Relation, plan: SortedBinaryUnion, workspace: UnionWorkspace,
               stream: CudaStream) -> None:
    """Merge and deduplicate sorted relations (union_cuda, lib.rs:1098-1177, plus PendingUnion::wait)."""
    L = _native.load()
    check_row_count(len(left))
    check_row_count(len(right))
    lf, ls = left.column(plan.left[0]), left.column(plan.left[1])
    rf, rs = right.column(plan.right[0]), right.column(plan.right[1])
    total = len(left) + len(right)
    ws = workspace
    ws.left = _grow_u64(ws.left, len(left))
    ws.right = _grow_u64(ws.right, len(right))
    ws.merged = _grow_u64(ws.merged, total)
    ws.unique = _grow_u64(ws.unique, total)
    out0 = _grow_u32(ws.output.columns[0], total)
    out1 = _grow_u32(ws.output.columns[1], total)
    ws.output = Relation(out0, out1, 0)
    temp_bytes = ctypes.c_size_t(0)
    _check("sparkalog_union_u32_temporary_bytes",
           L.sparkalog_union_u32_temporary_bytes(_ptr(ws.left), len(left), _ptr(ws.right), len(right),
                                                 _ptr(ws.merged), _ptr(ws.unique), _ptr(ws.count),
                                                 ctypes.byref(temp_bytes), stream.raw))
    temp = ws.temp.reserve(temp_bytes.value)
    _check("sparkalog_union_u32",
           L.sparkalog_union_u32(_ptr(lf), _ptr(ls), len(left), _ptr(rf), _ptr(rs), len(right), _ptr(ws.left),
                                 _ptr(ws.right), _ptr(ws.merged), _ptr(ws.unique), _ptr(ws.count), _ptr(out0),
                                 _ptr(out1), _ptr(temp), temp_bytes.value, stream.raw))
    ws.output.rows = _read_count(ws.count, stream)


def join_cuda(left: Relation, right: Relation, right_index: U32RangeIndex, plan: BinaryEqualityJoin,
              workspace: JoinWorkspace, stream: CudaStream) -> None:
    """Indexed equality join with count, scan and emit (join_cuda, lib.rs:1549-1648).

    As in the reference, one synchronisation separates the count stage from
    the emit stage so the output can be sized exactly."""
    L = _native.load()
    check_row_count(len(left))
    check_row_count(len(right))
    left_key = left.column(plan.left_key)
    right.column(plan.right_key)
    if len(right) != right_index.source_rows:
        raise IndexSourceMismatch(
            f"right relation has {len(right)} rows but its index has {right_index.source_rows}")
    proj = []
    for p in plan.output:
        src = left if p.input == JoinInput.LEFT else right
        proj.append((src.column(p.column), int(p.input)))
    n = len(left)
    ws = workspace
    ws.counts = _grow_u64(ws.counts, n)
    ws.offsets = _grow_u64(ws.offsets, n)
    temp_bytes = ctypes.c_size_t(0)
    _check("sparkalog_join_u32_temporary_bytes",
           L.sparkalog_join_u32_temporary_bytes(_ptr(ws.counts), _ptr(ws.offsets), n, ctypes.byref(temp_bytes),
                                                stream.raw))
    temp = ws.temp.reserve(temp_bytes.value)
    _check("sparkalog_join_u32_count",
           L.sparkalog_join_u32_count(_ptr(left_key), n, _ptr(right_index.keys), _ptr(right_index.starts),
                                      right_index.unique_keys, _ptr(ws.counts), _ptr(ws.offsets), _ptr(ws.total),
                                      _ptr(temp), temp_bytes.value, stream.raw))
    total = _read_count(ws.total, stream)
    out0 = _grow_u32(ws.output.columns[0], total)
    out1 = _grow_u32(ws.output.columns[1], total)
    _check("sparkalog_join_u32_emit",
           L.sparkalog_join_u32_emit(_ptr(left_key), n, _ptr(right_index.keys), _ptr(right_index.starts),
                                     _ptr(right_index.rows), right_index.unique_keys, _ptr(proj[0][0]), proj[0][1],
                                     _ptr(proj[1][0]), proj[1][1], _ptr(ws.offsets), _ptr(out0), _ptr(out1),
                                     stream.raw))
    stream.synchronize()
    ws.output = Relation(out0, out1, total)
