"""Binary-program execution on the device: the BinaryHybrid drop-in.

Mirrors ``BinaryProgramPlan`` / ``BinarySccPlan`` / ``BinarySeedPlan`` and
``execute_binary`` of crates/sparkalog-datalog/src/subset.rs:18-37,369-414,
and the backend choice of ``Database::run`` (database.rs:114-149): a program
that lowers to the binary subset runs here, on the GPU, every round of every
recursive SCC.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .recursion import RecursiveExecutor, RelationStore, SccSummary
from .relational import RecursiveSccPlan, RelationId


@dataclass(frozen=True)
class BinarySeedPlan:
    """subset.rs:18-23: target(x, y) :- source(..) projecting ``columns``."""

    target: RelationId
    source: RelationId
    columns: tuple[int, int]


@dataclass
class BinarySccPlan:
    """subset.rs:25-29."""

    plan: RecursiveSccPlan
    seeds: list[BinarySeedPlan] = field(default_factory=list)


@dataclass
class BinaryProgramPlan:
    """subset.rs:31-37."""

    predicate_count: int
    facts: list[tuple[RelationId, tuple[int, int]]] = field(default_factory=list)
    recursive_sccs: list[BinarySccPlan] = field(default_factory=list)
    outputs: list[RelationId] = field(default_factory=list)


@dataclass
class BinaryExecution:
    """subset.rs:364-367."""

    store: RelationStore
    summaries: list[SccSummary]


@dataclass(frozen=True)
class NegationClause:
    """``target(x, y) :- positive(x, y), !negative(x, y).`` — a non-recursive SCC
    with one seed clause whose negated atom reads a completed earlier stratum
    (general.rs:391-402,522-536)."""

    target: RelationId
    positive: RelationId
    negative: RelationId


@dataclass
class GeneralSccSummary:
    """GeneralSccSummary (general.rs:344-349): rows of each SCC relation,
    rounds executed and new rows; non-recursive SCCs report 1 round when they
    have a seed clause and 0 new rows (general.rs:400-402)."""

    relations: list[tuple[RelationId, int]]
    iterations: int
    new_rows: int


class ValueCatalog:
    """ValueCatalog (crates/sparkalog-datalog/src/catalog.rs:98-127) for u32 values, kept on
    the GPU: ``intern`` numbers unseen values by first appearance after the current size,
    ``decode`` maps ids back (Database::query's decode). Arrays may be NumPy (host) or
    CUDA tensors; results come back in the same kind."""

    def __init__(self, stream=None):
        import ctypes

        import torch

        from . import _native

        self._torch, self._ctypes, self._native = torch, ctypes, _native
        self._stream = stream if stream is not None else torch.cuda.current_stream()
        h = ctypes.c_void_p()
        self._check(_native.load().sparkalog_catalog_create(self._stream.cuda_stream, ctypes.byref(h)))
        self._h = h

    def _check(self, code: int) -> None:
        if code != 0:
            from .recursion import GenericExecutionError

            raise GenericExecutionError(code, self._native.last_error())

    def _call(self, fn, array):
        torch, ctypes = self._torch, self._ctypes
        if isinstance(array, torch.Tensor):
            out = torch.empty_like(array)
            fn(array.data_ptr(), array.numel(), 1, out.data_ptr())
            return out
        a = np.ascontiguousarray(np.asarray(array, dtype=np.uint32))
        out = np.empty_like(a)
        fn(a.ctypes.data if len(a) else None, len(a), 0, out.ctypes.data if len(a) else None)
        return out

    def intern(self, values):
        L, size = self._native.load(), self._ctypes.c_size_t(0)
        return self._call(lambda p, n, loc, o: self._check(
            L.sparkalog_catalog_intern_u32(self._h, p, n, loc, o, self._ctypes.byref(size))), values)

    def intern_rows(self, first, second):
        """Interns a binary relation row by row (Database::insert order: row[0], row[1], next row)."""
        torch = self._torch
        if isinstance(first, torch.Tensor):
            ids = self.intern(torch.stack([first, second], dim=1).reshape(-1))
            return ids[0::2].contiguous(), ids[1::2].contiguous()
        both = np.stack([np.asarray(first, dtype=np.uint32), np.asarray(second, dtype=np.uint32)], axis=1)
        ids = self.intern(both.reshape(-1))
        return ids[0::2].copy(), ids[1::2].copy()

    def decode(self, ids):
        L = self._native.load()
        return self._call(lambda p, n, loc, o: self._check(L.sparkalog_catalog_decode_u32(self._h, p, n, loc, o)),
                          ids)

    def __len__(self) -> int:
        size = self._ctypes.c_size_t(0)
        self._check(self._native.load().sparkalog_catalog_size(self._h, self._ctypes.byref(size)))
        return int(size.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._native.load().sparkalog_catalog_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pack(pairs: np.ndarray) -> np.ndarray:
    return (pairs[:, 0].astype(np.uint64) << np.uint64(32)) | pairs[:, 1].astype(np.uint64)


def _unpack(packed: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    return (packed >> np.uint64(32)).astype(np.uint32), (packed & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def execute_binary(plan: BinaryProgramPlan, max_iterations: int = 10_000, stream=None,
                   relations: dict[int, tuple[np.ndarray, np.ndarray]] | None = None) -> BinaryExecution:
    """execute_binary (subset.rs:369-414).

    Facts (plus optional bulk ``relations`` given as column pairs, the
    equivalent of many ``Database::insert`` calls) become one sorted,
    deduplicated set per relation (the reference's BTreeSet). Seed clauses
    project their source's set as it stands before any SCC runs. Recursive
    relations enter the store with FULL = DELTA = their set; the SCCs then run
    in order on the device.
    """
    sets: list[np.ndarray] = [np.zeros(0, dtype=np.uint64) for _ in range(plan.predicate_count)]
    by_rel: dict[int, list] = {}
    for rel, tup in plan.facts:
        by_rel.setdefault(rel.value, []).append(tup)
    for rel, tuples in by_rel.items():
        sets[rel] = np.unique(_pack(np.asarray(tuples, dtype=np.uint32).reshape(-1, 2)))
    for rel, (first, second) in (relations or {}).items():
        extra = (np.asarray(first, dtype=np.uint32).astype(np.uint64) << np.uint64(32)) | \
            np.asarray(second, dtype=np.uint32).astype(np.uint64)
        sets[rel] = np.unique(np.concatenate([sets[rel], extra]))
    for scc in plan.recursive_sccs:
        for seed in scc.seeds:
            first, second = _unpack(sets[seed.source.value])
            cols = (first, second)
            projected = (cols[seed.columns[0]].astype(np.uint64) << np.uint64(32)) | \
                cols[seed.columns[1]].astype(np.uint64)
            sets[seed.target.value] = np.unique(np.concatenate([sets[seed.target.value], projected]))
    recursive = {r.value for scc in plan.recursive_sccs for r in scc.plan.relations}
    store = RelationStore(stream)
    for rid, packed in enumerate(sets):
        cols = _unpack(packed)
        if rid in recursive:
            store.insert_recursive(rid, cols, cols)
        else:
            store.insert_static(rid, cols)
    summaries = []
    for scc in plan.recursive_sccs:
        executor = RecursiveExecutor.compile(scc.plan, store)
        summaries.append(executor.run(store, max_iterations))
        executor.close()
    return BinaryExecution(store, summaries)


def execute_stratified(predicate_count: int, strata: list, facts=None,
                       relations: dict[int, tuple[np.ndarray, np.ndarray]] | None = None,
                       max_iterations: int = 10_000, stream=None):
    """Runs a stratified binary program on the device, SCC by SCC in order.

    ``strata`` lists, in schedule order, ``BinarySccPlan`` entries (recursive
    SCCs: seeded from the facts, then iterated by the RecursiveExecutor) and
    ``NegationClause`` entries (evaluated with the store's anti-join against
    the completed FULL of the negated relation). Returns the store and one
    GeneralSccSummary per SCC, as execute_general does (general.rs:371-389).
    """
    plan = BinaryProgramPlan(predicate_count=predicate_count, facts=list(facts or []),
                             recursive_sccs=[s for s in strata if isinstance(s, BinarySccPlan)])
    sets: list[np.ndarray] = [np.zeros(0, dtype=np.uint64) for _ in range(predicate_count)]
    by_rel: dict[int, list] = {}
    for rel, tup in plan.facts:
        by_rel.setdefault(rel.value, []).append(tup)
    for rel, tuples in by_rel.items():
        sets[rel] = np.unique(_pack(np.asarray(tuples, dtype=np.uint32).reshape(-1, 2)))
    for rel, (first, second) in (relations or {}).items():
        extra = (np.asarray(first, dtype=np.uint32).astype(np.uint64) << np.uint64(32)) | \
            np.asarray(second, dtype=np.uint32).astype(np.uint64)
        sets[rel] = np.unique(np.concatenate([sets[rel], extra]))
    for scc in plan.recursive_sccs:
        for seed in scc.seeds:
            first, second = _unpack(sets[seed.source.value])
            cols = (first, second)
            projected = (cols[seed.columns[0]].astype(np.uint64) << np.uint64(32)) | \
                cols[seed.columns[1]].astype(np.uint64)
            sets[seed.target.value] = np.unique(np.concatenate([sets[seed.target.value], projected]))
    recursive = {r.value for scc in plan.recursive_sccs for r in scc.plan.relations}
    derived = {s.target.value for s in strata if isinstance(s, NegationClause)}
    store = RelationStore(stream)
    for rid, packed in enumerate(sets):
        if rid in derived:
            continue
        cols = _unpack(packed)
        if rid in recursive:
            store.insert_recursive(rid, cols, cols)
        else:
            store.insert_static(rid, cols)
    summaries = []
    for item in strata:
        if isinstance(item, BinarySccPlan):
            executor = RecursiveExecutor.compile(item.plan, store)
            s = executor.run(store, max_iterations)
            executor.close()
            summaries.append(GeneralSccSummary(s.relation_rows, s.iterations, s.total_new_rows))
        else:
            rows = store.anti_join(item.positive, item.negative, item.target)
            summaries.append(GeneralSccSummary([(item.target, rows)], 1, 0))
    return store, summaries
