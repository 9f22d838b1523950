"""Semi-naive fixpoint orchestration on the device (Tier B of the C ABI).

Mirrors crates/sparkalog-recursion/src/generic.rs: ``RelationStore``
(:16-121), ``RecursiveExecutor::{compile, run}`` (:407-525), ``SccSummary``
(:536-542), the ``GenericExecutionError`` / ``RelationStoreError`` variants and
``transitive_closure_scc`` (:629-661). The store keeps every relation resident
on the GPU; only explicit reads copy rows back.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .relational import (BinaryEqualityJoin, JoinInput, JoinProjection, RecursiveRulePlan, RecursiveSccPlan,
                         RelationId, path_join)

HOST, DEVICE = 0, 1
FULL, DELTA = 0, 1


class GenericExecutionError(RuntimeError):
    """Errors of RecursiveExecutor and RelationStore; ``kind`` names the reference's variant."""

    KINDS = {
        -1: "Missing", -2: "Duplicate", -3: "NotRecursive", -4: "EmptyScc", -5: "DuplicateSccRelation",
        -6: "DeltaOutsideScc", -7: "TargetOutsideScc", -8: "IncompatibleTargetPlans", -9: "MissingRuleTarget",
        -10: "IterationLimit", -11: "TooManyRows", -12: "MissingPlanColumn", -20: "DeviceFault",
        -21: "InvalidArgument", -22: "UnsortedFull", -23: "Load",
    }

    def __init__(self, code: int, message: str):
        self.code = code
        self.kind = self.KINDS.get(code, "Cuda" if code > 0 else f"Error{code}")
        super().__init__(f"{self.kind}: {message}")


RelationStoreError = GenericExecutionError


class LoadError(GenericExecutionError):
    """storage::LoadError (crates/sparkalog-storage/src/io.rs:7-20): ``kind`` is
    GitLfsPointer, InvalidFieldCount or InvalidU32, with the 1-based ``line`` and,
    for InvalidU32, the ``column`` and the field's text ``value``."""

    LOAD_KINDS = {1: "GitLfsPointer", 2: "InvalidFieldCount", 3: "InvalidU32",
                  # DelimitedError messages (ingest.rs:43-120), DatabaseError::Arity, a non-u32 value
                  4: "unterminated quoted field", 5: "expected delimiter after quoted field",
                  6: "empty fields are not values", 7: "record ends with an empty field", 8: "Arity", 9: "NotU32"}

    def __init__(self, code: int, message: str, kind: int, line: int, column: int, value: str | None):
        super().__init__(code, message)
        self.kind = self.LOAD_KINDS.get(kind, "Load")
        self.line, self.column, self.value = line, column, value


def _check(code: int) -> None:
    if code != 0:
        raise GenericExecutionError(code, _native.last_error())


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


@dataclass
class SccSummary:
    """SccSummary (generic.rs:536-542); every operator runs on the GPU, so placements are omitted."""

    iterations: int
    total_new_rows: int
    relation_rows: list[tuple[RelationId, int]]


class RelationStore:
    """Device-resident FULL/DELTA/NEWT buffers per relation (generic.rs:16-121)."""

    def __init__(self, stream: torch.cuda.Stream | None = None):
        L = _native.load()
        self._stream = stream if stream is not None else torch.cuda.current_stream()
        h = ctypes.c_void_p()
        _check(L.sparkalog_store_create(self._stream.cuda_stream, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        h, self._h = getattr(self, "_h", None), None
        if h:
            _native.load().sparkalog_store_destroy(h)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @staticmethod
    def _columns(relation):
        """Accepts (first, second) host arrays or device tensors; returns (p0, p1, rows, location, keep)."""
        first, second = relation
        if isinstance(first, torch.Tensor) and first.is_cuda:
            if first.dtype not in (torch.int32, torch.uint32) or not first.is_contiguous():
                raise ValueError("device columns must be contiguous 32-bit tensors")
            return first.data_ptr(), second.data_ptr(), int(first.numel()), DEVICE, (first, second)
        a, b = _u32(first), _u32(second)
        if len(a) != len(b):
            raise ValueError("column lengths differ")
        return a.ctypes.data, b.ctypes.data, len(a), HOST, (a, b)

    def insert_static(self, rid: RelationId | int, relation) -> None:
        """RelationStore::insert_static (generic.rs:36-51)."""
        p0, p1, n, loc, keep = self._columns(relation)
        _check(_native.load().sparkalog_store_insert_static(self._h, int(getattr(rid, "value", rid)), p0, p1, n, loc))
        del keep

    def insert_recursive(self, rid: RelationId | int, full, delta) -> None:
        """RelationStore::insert_recursive (generic.rs:53-79)."""
        f0, f1, fn, loc, keep_f = self._columns(full)
        d0, d1, dn, loc_d, keep_d = self._columns(delta)
        if loc != loc_d:
            raise ValueError("FULL and DELTA must both be host arrays or both device tensors")
        _check(_native.load().sparkalog_store_insert_recursive(self._h, int(getattr(rid, "value", rid)), f0, f1, fn,
                                                               d0, d1, dn, loc))
        del keep_f, keep_d

    def rows(self, rid: RelationId | int, version: int = FULL) -> int:
        n = ctypes.c_size_t(0)
        _check(_native.load().sparkalog_store_rows(self._h, int(getattr(rid, "value", rid)), version, ctypes.byref(n)))
        return int(n.value)

    def _read(self, rid, version: int) -> tuple[np.ndarray, np.ndarray]:
        n = self.rows(rid, version)
        a = np.empty(max(n, 1), dtype=np.uint32)
        b = np.empty(max(n, 1), dtype=np.uint32)
        _check(_native.load().sparkalog_store_read(self._h, int(getattr(rid, "value", rid)), version, a.ctypes.data,
                                                   b.ctypes.data, HOST))
        return a[:n], b[:n]

    def full(self, rid: RelationId | int) -> tuple[np.ndarray, np.ndarray]:
        """RelationStore::full (generic.rs:81-83), copied to the host as two columns."""
        return self._read(rid, FULL)

    def delta(self, rid: RelationId | int) -> tuple[np.ndarray, np.ndarray]:
        """RelationStore::delta (generic.rs:85-91)."""
        return self._read(rid, DELTA)

    def anti_join(self, left: RelationId | int, right: RelationId | int, out: RelationId | int) -> int:
        """Stores ``out(x, y) :- left(x, y), !right(x, y).`` as a new static relation
        (GeneralCpu's clause evaluation, general.rs:478-551); returns its row count."""
        ids = [int(getattr(r, "value", r)) for r in (left, right, out)]
        _check(_native.load().sparkalog_store_anti_join(self._h, *ids))
        return self.rows(ids[2])

    def compact(self, rid: RelationId | int) -> None:
        """Merges FULL's levels into one sorted run on the device (the single
        sorted FULL the reference's TargetRuntime::apply keeps, generic.rs:360-397)."""
        _check(_native.load().sparkalog_store_compact(self._h, int(getattr(rid, "value", rid))))

    def drop(self, rid: RelationId | int) -> None:
        """Removes a relation and frees its device memory."""
        _check(_native.load().sparkalog_store_drop(self._h, int(getattr(rid, "value", rid))))

    def has(self, rid: RelationId | int) -> bool:
        n = ctypes.c_size_t(0)
        return _native.load().sparkalog_store_rows(self._h, int(getattr(rid, "value", rid)), FULL,
                                                   ctypes.byref(n)) == 0

    def select(self, rid: RelationId | int, out: RelationId | int, where=(None, None), same: bool = False,
               project=(0, 1)) -> int:
        """out = {(c0, c1)} over the rows (x, y) of FULL(rid) with x == where[0] and
        y == where[1] (each when not None) and x == y when ``same``; each output
        column is ``0`` (x), ``1`` (y) or ``("const", value)``. Returns |out|."""
        sp = _native.SelectC()
        sp.where_mask = (1 if where[0] is not None else 0) | (2 if where[1] is not None else 0) | (4 if same else 0)
        sp.where_value[0] = where[0] or 0
        sp.where_value[1] = where[1] or 0
        for k, src in enumerate(project):
            if isinstance(src, tuple):
                sp.out_source[k], sp.out_value[k] = 2, int(src[1])
            else:
                sp.out_source[k] = int(src)
        n = ctypes.c_size_t(0)
        _check(_native.load().sparkalog_store_select(self._h, int(getattr(rid, "value", rid)), ctypes.byref(sp),
                                                     int(getattr(out, "value", out)), ctypes.byref(n)))
        return int(n.value)

    def join(self, left: RelationId | int, right: RelationId | int, left_key: int, right_key: int,
             projection, out: RelationId | int) -> int:
        """out = distinct projection of left ⋈ right on left[left_key] == right[right_key];
        ``projection`` is ((side, column), (side, column)) with side 0 = left, 1 = right."""
        sides = _u32([projection[0][0], projection[1][0]])
        cols = _u32([projection[0][1], projection[1][1]])
        n = ctypes.c_size_t(0)
        _check(_native.load().sparkalog_store_join(self._h, int(getattr(left, "value", left)),
                                                   int(getattr(right, "value", right)), left_key, right_key,
                                                   sides.ctypes.data_as(_native.c_u32p),
                                                   cols.ctypes.data_as(_native.c_u32p),
                                                   int(getattr(out, "value", out)), ctypes.byref(n)))
        return int(n.value)

    def load_binary_u32(self, rid: RelationId | int, text, recursive: bool = False) -> int:
        """Parses whitespace-separated u32 pairs on the GPU and inserts them as relation
        ``rid`` (load_binary_u32, crates/sparkalog-storage/src/io.rs:72-141); ``text``
        is bytes, str, or a uint8 CUDA tensor. Returns the number of rows read."""
        L = _native.load()
        if isinstance(text, str):
            text = text.encode()
        if isinstance(text, torch.Tensor):
            ptr, nbytes, loc, host = text.data_ptr(), int(text.numel()), DEVICE, None
        else:
            # bytes-like or a uint8 NumPy array (e.g. a pinned buffer): read in place.
            host = text if isinstance(text, np.ndarray) else np.frombuffer(text, dtype=np.uint8)
            host = np.ascontiguousarray(host.view(np.uint8).reshape(-1))
            ptr, nbytes, loc = host.ctypes.data if len(host) else None, len(host), HOST
        rows = ctypes.c_size_t(0)
        err = _native.LoadErrorC()
        code = L.sparkalog_store_load_binary_u32(self._h, int(getattr(rid, "value", rid)), ptr, nbytes, loc,
                                                 1 if recursive else 0, ctypes.byref(rows), ctypes.byref(err))
        if code == -23:
            value = None
            if err.kind == 3:
                raw = host if host is not None else text.cpu().numpy()
                value = bytes(raw[err.field_offset:err.field_offset + err.field_length]).decode(errors="replace")
            raise LoadError(code, _native.last_error(), err.kind, int(err.line), int(err.column), value)
        _check(code)
        return int(rows.value)

    def load_delimited_u32(self, rid: RelationId | int, text, delimiter: str = ",", has_header: bool = False,
                           recursive: bool = False) -> int:
        """Database::load_delimited (database.rs:165-177) for a binary relation of u32
        values, parsed on the GPU; ``text`` is bytes, str, or a uint8 CUDA tensor.
        Returns the number of rows read. Errors raise LoadError with the reference's
        line, byte column and message (``kind``)."""
        L = _native.load()
        if isinstance(text, str):
            text = text.encode()
        if isinstance(text, torch.Tensor):
            ptr, nbytes, loc, host = text.data_ptr(), int(text.numel()), DEVICE, None
        else:
            host = text if isinstance(text, np.ndarray) else np.frombuffer(text, dtype=np.uint8)
            host = np.ascontiguousarray(host.view(np.uint8).reshape(-1))
            ptr, nbytes, loc = host.ctypes.data if len(host) else None, len(host), HOST
        d = delimiter.encode()
        if len(d) != 1:
            raise ValueError("the delimiter is one byte")
        rows = ctypes.c_size_t(0)
        err = _native.LoadErrorC()
        code = L.sparkalog_store_load_delimited_u32(self._h, int(getattr(rid, "value", rid)), ptr, nbytes, loc, d[0],
                                                    1 if has_header else 0, 1 if recursive else 0,
                                                    ctypes.byref(rows), ctypes.byref(err))
        if code == -23:
            value = None
            if err.kind == 9:
                raw = host if host is not None else text.cpu().numpy()
                value = bytes(raw[err.field_offset:err.field_offset + err.field_length]).decode(errors="replace")
            raise LoadError(code, _native.last_error(), err.kind, int(err.line), int(err.column), value)
        _check(code)
        return int(rows.value)

    def load_delimited(self, rid: RelationId | int, text, catalog, delimiter: str = ",", has_header: bool = False,
                       recursive: bool = False) -> int:
        """Database::load_delimited (database.rs:165-177) for a binary relation of any
        values (U32, String, Symbol), parsed and interned into ``catalog`` (a
        datalog.ValueCatalog) on the GPU; the relation holds value ids. Returns the
        number of rows read; errors raise LoadError as load_delimited_u32."""
        L = _native.load()
        if isinstance(text, str):
            text = text.encode()
        if isinstance(text, torch.Tensor):
            ptr, nbytes, loc = text.data_ptr(), int(text.numel()), DEVICE
        else:
            host = text if isinstance(text, np.ndarray) else np.frombuffer(text, dtype=np.uint8)
            host = np.ascontiguousarray(host.view(np.uint8).reshape(-1))
            ptr, nbytes, loc = host.ctypes.data if len(host) else None, len(host), HOST
        d = delimiter.encode()
        if len(d) != 1:
            raise ValueError("the delimiter is one byte")
        rows = ctypes.c_size_t(0)
        err = _native.LoadErrorC()
        code = L.sparkalog_store_load_delimited_values(self._h, catalog.handle, int(getattr(rid, "value", rid)), ptr,
                                                       nbytes, loc, d[0], 1 if has_header else 0,
                                                       1 if recursive else 0, ctypes.byref(rows), ctypes.byref(err))
        if code == -23:
            raise LoadError(code, _native.last_error(), err.kind, int(err.line), int(err.column), None)
        _check(code)
        return int(rows.value)

    def append(self, rid: RelationId | int, relation) -> None:
        """FULL u= rows (and DELTA u= the genuinely new rows of a recursive relation),
        so a resident fixpoint continues from them."""
        p0, p1, n, loc, keep = self._columns(relation)
        _check(_native.load().sparkalog_store_append(self._h, int(getattr(rid, "value", rid)), p0, p1, n, loc))
        del keep

    def extract_segment(self, rid: RelationId | int, shift: int, segment: int, untag: bool = False,
                        device: bool = False):
        """Sorted rows of FULL whose first column >> shift == segment; with
        ``untag`` the segment bits of both columns are cleared on the device.
        Host numpy columns, or with ``device`` two int32 CUDA tensors (the u32
        bits) allocated on the store's stream."""
        L = _native.load()
        rid = int(getattr(rid, "value", rid))
        n = ctypes.c_size_t(0)
        loc = DEVICE if device else HOST
        if untag:
            call = lambda a, b: L.sparkalog_store_extract_segment_untagged(self._h, rid, shift, segment, 1, a, b, loc,
                                                                            ctypes.byref(n))
        else:
            call = lambda a, b: L.sparkalog_store_extract_segment(self._h, rid, shift, segment, a, b, loc,
                                                                  ctypes.byref(n))
        _check(call(None, None))
        if device:
            with torch.cuda.stream(self._stream):
                a = torch.empty(max(n.value, 1), dtype=torch.int32, device="cuda")
                b = torch.empty(max(n.value, 1), dtype=torch.int32, device="cuda")
            _check(call(a.data_ptr(), b.data_ptr()))
            return a[: n.value], b[: n.value]
        a = np.empty(max(n.value, 1), dtype=np.uint32)
        b = np.empty(max(n.value, 1), dtype=np.uint32)
        _check(call(a.ctypes.data, b.ctypes.data))
        return a[: n.value], b[: n.value]

    @property
    def stream(self):
        return self._stream

    def remove_segments(self, rid: RelationId | int, shift: int, segments) -> None:
        """Drops every row whose first column >> shift is in ``segments`` from FULL and DELTA."""
        segs = _u32(list(segments))
        _check(_native.load().sparkalog_store_remove_segments(self._h, int(getattr(rid, "value", rid)), shift,
                                                              segs.ctypes.data_as(_native.c_u32p), len(segs)))

    def read_into(self, rid: RelationId | int, version: int, first, second) -> int:
        """Copies FULL/DELTA into caller buffers (numpy host arrays, possibly pinned, or device tensors)."""
        n = self.rows(rid, version)
        if isinstance(first, torch.Tensor) and first.is_cuda:
            p0, p1, loc = first.data_ptr(), second.data_ptr(), DEVICE
        elif isinstance(first, torch.Tensor):
            p0, p1, loc = first.data_ptr(), second.data_ptr(), HOST
        else:
            p0, p1, loc = first.ctypes.data, second.ctypes.data, HOST
        _check(_native.load().sparkalog_store_read(self._h, int(getattr(rid, "value", rid)), version, p0, p1, loc))
        return n


def _rule_c(rule: RecursiveRulePlan) -> _native.RulePlanC:
    c = _native.RulePlanC()
    c.target = rule.target.value
    c.delta_input = rule.delta_input.value
    c.right_input = rule.right_input.value
    c.left_key = rule.join.left_key
    c.right_key = rule.join.right_key
    for j, p in enumerate(rule.join.output):
        c.proj_side[j] = int(p.input)
        c.proj_col[j] = p.column
    c.distinct_cols[:] = list(rule.distinct.columns)
    c.anti_left[:] = list(rule.anti_join.left)
    c.anti_right[:] = list(rule.anti_join.right)
    c.union_left[:] = list(rule.union.left)
    c.union_right[:] = list(rule.union.right)
    return c


class RecursiveExecutor:
    """RecursiveExecutor (generic.rs:400-525)."""

    def __init__(self, handle: ctypes.c_void_p, plan: RecursiveSccPlan):
        self._h = handle
        self.plan = plan

    @classmethod
    def compile(cls, plan: RecursiveSccPlan, store: RelationStore) -> "RecursiveExecutor":
        """RecursiveExecutor::compile (generic.rs:407-470)."""
        rel = _u32([r.value for r in plan.relations])
        rules = (_native.RulePlanC * max(len(plan.rules), 1))(*[_rule_c(r) for r in plan.rules])
        h = ctypes.c_void_p()
        _check(_native.load().sparkalog_executor_compile(store.handle, rel.ctypes.data_as(_native.c_u32p), len(rel),
                                                         rules, len(plan.rules), ctypes.byref(h)))
        ex = cls(h, plan)
        # The autotuner's saved choice for this device, when there is one.
        from . import autotune

        tuned = autotune.saved_tuning()
        if tuned is not None:
            ex.set_tuning(tuned)
        return ex

    def close(self) -> None:
        h, self._h = getattr(self, "_h", None), None
        if h:
            _native.load().sparkalog_executor_destroy(h)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, store: RelationStore, max_iterations: int = 10_000) -> SccSummary:
        """RecursiveExecutor::run (generic.rs:472-516): loops while any DELTA of the SCC is
        non-empty and counts every executed round."""
        n = len(self.plan.relations)
        ids = (ctypes.c_uint32 * max(n, 1))()
        rows = (ctypes.c_uint64 * max(n, 1))()
        s = _native.SccSummaryC()
        s.relation_count = n
        s.relation_ids = ids
        s.relation_rows = rows
        _check(_native.load().sparkalog_executor_run(self._h, store.handle, max_iterations, ctypes.byref(s)))
        return SccSummary(int(s.iterations), int(s.total_new_rows),
                          [(RelationId(int(ids[i])), int(rows[i])) for i in range(n)])


    def step(self, store: RelationStore, rounds: int = 1) -> tuple[SccSummary, bool]:
        """Runs at most ``rounds`` rounds (no error at the limit); returns the
        summary of those rounds and whether every DELTA is now empty."""
        n = len(self.plan.relations)
        ids = (ctypes.c_uint32 * max(n, 1))()
        rows = (ctypes.c_uint64 * max(n, 1))()
        s = _native.SccSummaryC()
        s.relation_count = n
        s.relation_ids = ids
        s.relation_rows = rows
        conv = ctypes.c_int(0)
        _check(_native.load().sparkalog_executor_step(self._h, store.handle, rounds, ctypes.byref(s),
                                                      ctypes.byref(conv)))
        return (SccSummary(int(s.iterations), int(s.total_new_rows),
                           [(RelationId(int(ids[i])), int(rows[i])) for i in range(n)]), bool(conv.value))

    def track_segments(self, shift: int, count: int) -> None:
        """Records per-segment (first column >> shift) activity each round; see segment_stats."""
        _check(_native.load().sparkalog_executor_track_segments(self._h, shift, count))
        self._segments = count

    def segment_stats(self) -> tuple[np.ndarray, np.ndarray]:
        """(last_active_round, new_rows) per segment: a segment that gained rows in
        round r (0-based) has last_active_round >= r + 1."""
        n = getattr(self, "_segments", 0)
        seen = np.zeros(max(n, 1), dtype=np.uint32)
        new = np.zeros(max(n, 1), dtype=np.uint64)
        _check(_native.load().sparkalog_executor_segment_stats(self._h, seen.ctypes.data_as(_native.c_u32p),
                                                               new.ctypes.data_as(_native.c_u64p)))
        return seen[:n], new[:n]

    def set_profiling(self, enable: bool) -> None:
        """Times every kernel class with CUDA events on the store's stream."""
        _check(_native.load().sparkalog_executor_set_profiling(self._h, 1 if enable else 0))

    def set_fused(self, enable: bool) -> None:
        """Enables (default) or disables the fused join + distinct kernel; results are identical."""
        _check(_native.load().sparkalog_executor_set_fused(self._h, 1 if enable else 0))

    def trace(self, reset: bool = False) -> list[dict]:
        """Per-round operator cardinalities (delta, join, unique, new and FULL rows)."""
        L = _native.load()
        n = ctypes.c_size_t(0)
        _check(L.sparkalog_executor_trace(self._h, None, 0, ctypes.byref(n), 0))
        buf = (_native.RoundTraceC * max(n.value, 1))()
        _check(L.sparkalog_executor_trace(self._h, buf, n.value, ctypes.byref(n), 1 if reset else 0))
        return [{f: int(getattr(buf[i], f)) for f, _ in _native.RoundTraceC._fields_} for i in range(n.value)]

    def set_member_set(self, enable: bool) -> None:
        """Enables or disables (default) FULL's hash set for the anti-join; results are identical."""
        _check(_native.load().sparkalog_executor_set_member_set(self._h, 1 if enable else 0))

    def set_device_loop(self, enable: bool) -> None:
        """Enables (default) or disables device-driven tail rounds; results are identical."""
        _check(_native.load().sparkalog_executor_set_device_loop(self._h, 1 if enable else 0))

    def device_loop_stats(self) -> tuple[int, int]:
        """(graph launches, rounds applied) of the device-driven loop over the executor's lifetime."""
        a, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
        _check(_native.load().sparkalog_executor_device_loop_stats(self._h, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def tuning(self) -> dict:
        """The executor's launch shapes and thresholds (sparkalog_tuning)."""
        t = _native.TuningC()
        _check(_native.load().sparkalog_executor_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, tuning: dict) -> None:
        """Replaces some or all tuning values; results are identical for every valid value."""
        t = _native.TuningC()
        _check(_native.load().sparkalog_executor_get_tuning(self._h, ctypes.byref(t)))
        for name, value in tuning.items():
            if name not in dict(_native.TuningC._fields_):
                raise KeyError(f"unknown tuning value {name!r}")
            setattr(t, name, int(value))
        _check(_native.load().sparkalog_executor_set_tuning(self._h, ctypes.byref(t)))

    def stats(self, reset: bool = False) -> dict:
        """Per-kernel-class launches, milliseconds and algorithmic bytes, plus total launches."""
        s = _native.KernelStatsC()
        _check(_native.load().sparkalog_executor_stats(self._h, ctypes.byref(s), 1 if reset else 0))
        classes = {name: {"launches": int(s.launches[i]), "ms": float(s.milliseconds[i]),
                          "bytes": float(s.bytes[i])} for i, name in enumerate(_native.KERNEL_CLASSES)}
        return {"classes": classes, "total_launches": int(s.total_launches), "rounds": int(s.rounds)}


def reserve_device_memory(nbytes: int, stream: torch.cuda.Stream | None = None) -> None:
    """Grows and keeps the device memory pool that relations are allocated from."""
    s = stream if stream is not None else torch.cuda.current_stream()
    _check(_native.load().sparkalog_reserve_device_memory(int(nbytes), s.cuda_stream))


def transitive_closure_scc(path: RelationId, edge: RelationId) -> RecursiveSccPlan:
    """transitive_closure_scc (generic.rs:629-661)."""
    return RecursiveSccPlan(relations=[path],
                            rules=[RecursiveRulePlan(target=path, delta_input=path, right_input=edge,
                                                     join=path_join())])


__all__ = [
    "GenericExecutionError", "RelationStoreError", "RelationStore", "RecursiveExecutor", "SccSummary",
    "transitive_closure_scc", "BinaryEqualityJoin", "JoinInput", "JoinProjection", "FULL", "DELTA",
]
