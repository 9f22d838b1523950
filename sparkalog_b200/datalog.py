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


@dataclass(frozen=True)
class PlannedAtom:
    """PlannedAtom (crates/sparkalog-relational/src/lib.rs:104-109) of a binary
    predicate: each term is ``("b", id)``, a binding, or ``("v", value)``, a
    constant (an interned value id)."""

    relation: RelationId
    terms: tuple


@dataclass(frozen=True)
class GeneralClause:
    """A non-recursive clause (RelationalClausePlan, relational/src/lib.rs:113-121):
    ``target(head) :- positive..., !negative...``, evaluated on the device."""

    target: RelationId
    head: tuple
    positive: tuple
    negative: tuple = ()


@dataclass(frozen=True)
class NonRecursiveScc:
    """A non-recursive SCC of a stratified program: every clause deriving
    ``target`` (general.rs:391-402 evaluates them once, in order, and unions
    their outputs)."""

    target: RelationId
    clauses: tuple


class UnsupportedClause(ValueError):
    """A clause shape the device lowering does not take (see evaluate_clause)."""


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

    @property
    def handle(self):
        return self._h

    def values(self) -> list[tuple]:
        """Every interned value in id order, as ("u32", n), ("string", s) or
        ("symbol", s) (InternedValue, catalog.rs:10-14), read from the device."""
        ctypes, L = self._ctypes, self._native.load()
        n = len(self)
        used = ctypes.c_size_t(0)
        self._check(L.sparkalog_catalog_export(self._h, None, None, None, None, 0, ctypes.byref(used)))
        kinds = np.zeros(max(n, 1), dtype=np.uint32)
        numbers = np.zeros(max(n, 1), dtype=np.uint32)
        offsets = np.zeros(n + 1, dtype=np.uint64)
        raw = np.zeros(max(used.value, 1), dtype=np.uint8)
        self._check(L.sparkalog_catalog_export(self._h, kinds.ctypes.data_as(self._native.c_u32p),
                                               numbers.ctypes.data_as(self._native.c_u32p),
                                               offsets.ctypes.data_as(self._native.c_u64p), raw.ctypes.data,
                                               len(raw), ctypes.byref(used)))
        out = []
        for i in range(n):
            if kinds[i] == 0:
                out.append(("u32", int(numbers[i])))
            else:
                text = bytes(raw[int(offsets[i]):int(offsets[i + 1])]).decode()
                out.append(("string" if kinds[i] == 1 else "symbol", text))
        return out

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
    SCCs: seeded from the facts, then iterated by the RecursiveExecutor),
    ``NegationClause`` entries (evaluated with the store's anti-join against
    the completed FULL of the negated relation) and ``NonRecursiveScc``
    entries (general non-recursive clauses: constants, repeated bindings,
    joins of two atoms, head constants, negated atoms; see evaluate_clause). Returns the store and one
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
    derived |= {s.target.value for s in strata if isinstance(s, NonRecursiveScc) and len(sets[s.target.value]) == 0}
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
        elif isinstance(item, NonRecursiveScc):
            summaries.append(evaluate_nonrecursive(store, item))
        else:
            rows = store.anti_join(item.positive, item.negative, item.target)
            summaries.append(GeneralSccSummary([(item.target, rows)], 1, 0))
    return store, summaries


# Relation ids at and above this are the clause evaluator's temporaries.
_TEMP_BASE = 1 << 30


class _Temps:
    def __init__(self, store: RelationStore):
        self.store = store
        self.next = _TEMP_BASE
        self.live: list[int] = []

    def new(self) -> int:
        self.next += 1
        self.live.append(self.next)
        return self.next

    def drop_all(self, keep=()) -> None:
        for t in self.live:
            if t not in keep and self.store.has(t):
                self.store.drop(t)
        self.live = [t for t in self.live if t in keep]


def _bindings(atom: PlannedAtom) -> dict:
    """binding id -> the first column that binds it."""
    out = {}
    for col, (kind, x) in enumerate(atom.terms):
        if kind == "b" and x not in out:
            out[x] = col
    return out


def _atom_filter(atom: PlannedAtom):
    """(where, same) of an atom: constants compared, a repeated binding equal."""
    where = [None, None]
    for col, (kind, x) in enumerate(atom.terms):
        if kind == "v":
            where[col] = int(x)
    same = (atom.terms[0][0] == "b" and atom.terms[1][0] == "b" and atom.terms[0][1] == atom.terms[1][1])
    return tuple(where), same


def evaluate_clause(store: RelationStore, clause: GeneralClause, temps: _Temps) -> int:
    """Evaluates one non-recursive binary clause on the device (general.rs:478-551)
    into a new temporary relation and returns its id.

    Taken: one positive atom, or two that share exactly one binding; constants
    and repeated bindings in positive atoms and constants in the head; negated
    atoms whose two bindings are the head's two bindings (in either order).
    Other shapes raise UnsupportedClause (GeneralCpu evaluates them)."""
    pos = list(clause.positive)
    for atom in pos + list(clause.negative):
        if len(atom.terms) != 2:
            raise UnsupportedClause("binary predicates only")
    if len(clause.head) != 2:
        raise UnsupportedClause("binary predicates only")
    if len(pos) == 1:
        a = pos[0]
        where, same = _atom_filter(a)
        cols = _bindings(a)
        project = []
        for kind, x in clause.head:
            if kind == "v":
                project.append(("const", int(x)))
            elif x in cols:
                project.append(cols[x])
            else:
                raise UnsupportedClause("head binding not bound by a positive atom")
        out = temps.new()
        store.select(a.relation, out, where, same, tuple(project))
    elif len(pos) == 2:
        a, b = pos
        ca, cb = _bindings(a), _bindings(b)
        shared = sorted(set(ca) & set(cb))
        if len(shared) != 1:
            raise UnsupportedClause("two positive atoms must share exactly one binding")
        z = shared[0]
        inputs = []
        for atom in (a, b):
            where, same = _atom_filter(atom)
            if where != (None, None) or same:
                t = temps.new()
                store.select(atom.relation, t, where, same, (0, 1))
                inputs.append(t)
            else:
                inputs.append(atom.relation)
        projection, post, consts = [], [], False
        for kind, x in clause.head:
            if kind == "v":
                projection.append((0, ca[z]))
                post.append(("const", int(x)))
                consts = True
            elif x in ca:
                projection.append((0, ca[x]))
                post.append(len(post))
            elif x in cb:
                projection.append((1, cb[x]))
                post.append(len(post))
            else:
                raise UnsupportedClause("head binding not bound by a positive atom")
        out = temps.new()
        store.join(inputs[0], inputs[1], ca[z], cb[z], tuple(projection), out)
        if consts:
            t = temps.new()
            store.select(out, t, (None, None), False, tuple(post))
            out = t
    else:
        raise UnsupportedClause("one or two positive atoms")
    head = [x if kind == "b" else None for kind, x in clause.head]
    for n in clause.negative:
        kinds = [k for k, _ in n.terms]
        ids = [x for _, x in n.terms]
        if kinds != ["b", "b"] or None in head:
            raise UnsupportedClause("a negated atom must bind the head's two bindings")
        if ids == head:
            right = n.relation
        elif ids == head[::-1]:
            right = temps.new()
            store.select(n.relation, right, (None, None), False, (1, 0))
        else:
            raise UnsupportedClause("a negated atom must bind the head's two bindings")
        t = temps.new()
        store.anti_join(out, right, t)
        out = t
    return out


def evaluate_nonrecursive(store: RelationStore, scc: NonRecursiveScc) -> GeneralSccSummary:
    """Every clause of a non-recursive SCC, unioned into its target (which may
    already hold facts); GeneralCpu's summary for it: 1 round when it has a
    clause, 0 new rows (general.rs:391-402)."""
    temps = _Temps(store)
    try:
        results = [evaluate_clause(store, c, temps) for c in scc.clauses]
        target = scc.target.value
        for k, t in enumerate(results):
            if not store.has(target):
                store.select(t, target, (None, None), False, (0, 1))
                continue
            n = store.rows(t)
            if n:
                import torch

                cols = (torch.empty(n, dtype=torch.int32, device="cuda"),
                        torch.empty(n, dtype=torch.int32, device="cuda"))
                store.read_into(t, 0, cols[0], cols[1])
                store.append(target, cols)
        if not store.has(target):
            empty = np.zeros(0, dtype=np.uint32)
            store.insert_static(target, (empty, empty))
    finally:
        temps.drop_all()
    return GeneralSccSummary([(scc.target, store.rows(scc.target))], 1 if scc.clauses else 0, 0)
