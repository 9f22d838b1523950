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
