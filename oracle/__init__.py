"""CPU oracle for the sparkalog binary recursive operator pipeline.

TEST INFRASTRUCTURE ONLY: the reference the CUDA path is compared against. Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package; the product package never does.

``liboracle.so`` (built from ``oracle.cpp`` by ``oracle/Makefile``) restates
the reference's CPU operators and semi-naive loop; this module wraps it and
adds two pure-Python restatements for small inputs:

* ``execute_binary`` — the seeding of ``crates/sparkalog-datalog/src/subset.rs:369-414``;
* ``general_cpu`` — the nested-loop ``GeneralCpu`` evaluator of
  ``crates/sparkalog-datalog/src/general.rs:371-551`` (strata, SCC loop,
  negation against a completed FULL), the reference's only evaluator for
  stratified negation.

Parity is pinned by the reference's own known-answer tests (restated in
``tests/golden/``), because the Rust reference cannot be compiled here (no
cargo or rustc). ``oracle/_ref/libsparkalog_reference_cuda.so`` is the
reference's own ``column_ops.cu`` compiled unmodified for sm_100a by
``make -C oracle reference``; GPU tests use it as a second, independent check
of the operator ABI when it is present.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "liboracle.so"
REF_CUDA_PATH = ORACLE_DIR / "_ref" / "libsparkalog_reference_cuda.so"

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)


class OracleRulePlan(ctypes.Structure):
    """Flat RecursiveRulePlan (crates/sparkalog-relational/src/lib.rs:74-82)."""

    _fields_ = [
        ("target", ctypes.c_uint32),
        ("delta_input", ctypes.c_uint32),
        ("right_input", ctypes.c_uint32),
        ("left_key", ctypes.c_uint32),
        ("right_key", ctypes.c_uint32),
        ("proj_side", ctypes.c_uint32 * 2),
        ("proj_col", ctypes.c_uint32 * 2),
        ("distinct_cols", ctypes.c_uint32 * 2),
        ("anti_left", ctypes.c_uint32 * 2),
        ("anti_right", ctypes.c_uint32 * 2),
        ("union_left", ctypes.c_uint32 * 2),
        ("union_right", ctypes.c_uint32 * 2),
    ]


def reference_root() -> Path:
    """The reference checkout: $SPARKALOG_REFERENCE, else a directory named
    ``reference`` beside this repository's root (the Makefile's default)."""
    env = os.environ.get("SPARKALOG_REFERENCE")
    return Path(env) if env else ORACLE_DIR.parent.parent / "reference"


def build() -> None:
    """Compiles liboracle.so (and the reference CUDA library when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "liboracle.so"], check=True)
    ref = reference_root()
    if (ref / "crates/sparkalog-execution/native/column_ops.cu").exists():
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "reference", f"REFERENCE={ref}"], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.oracle_load_binary_u32.restype = ctypes.c_int
        L.oracle_load_binary_u32.argtypes = [ctypes.c_char_p, ctypes.c_uint64, _u32p, _u32p, ctypes.c_uint64,
                                             ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                             ctypes.POINTER(ctypes.c_int)]
        L.oracle_intern_u32.restype = None
        L.oracle_intern_u32.argtypes = [_u32p, ctypes.c_uint64, _u32p]
        L.oracle_general_tc.restype = ctypes.c_int
        L.oracle_general_tc.argtypes = [_u32p, _u32p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                        ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_int)]
        L.oracle_splitmix64.restype = ctypes.c_uint64
        L.oracle_splitmix64.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_er_edges.restype = ctypes.c_uint64
        L.oracle_er_edges.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _u32p, _u32p]
        L.oracle_range_index_build.restype = ctypes.c_uint64
        L.oracle_range_index_build.argtypes = [_u32p, ctypes.c_uint64, _u32p, _u32p, _u32p]
        L.oracle_join_count.restype = ctypes.c_uint64
        L.oracle_join_count.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p, _u32p, ctypes.c_uint64,
                                        ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_join.restype = ctypes.c_uint64
        L.oracle_join.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p, _u32p, ctypes.c_uint64, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.c_int, _u32p, _u32p]
        L.oracle_distinct.restype = ctypes.c_uint64
        L.oracle_distinct.argtypes = [_u32p, _u32p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_int, _u32p, _u32p]
        for name in ("oracle_anti_join", "oracle_union"):
            f = getattr(L, name)
            f.restype = ctypes.c_uint64
            f.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p, _u32p, ctypes.c_uint64, ctypes.c_int, _u32p, _u32p]
        L.oracle_store_new.restype = ctypes.c_void_p
        L.oracle_store_free.argtypes = [ctypes.c_void_p]
        L.oracle_store_insert_static.restype = ctypes.c_int
        L.oracle_store_insert_static.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint64]
        L.oracle_store_insert_recursive.restype = ctypes.c_int
        L.oracle_store_insert_recursive.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _u32p, _u32p,
                                                    ctypes.c_uint64, _u32p, _u32p, ctypes.c_uint64]
        L.oracle_store_len.restype = ctypes.c_uint64
        L.oracle_store_len.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int]
        L.oracle_store_copy.restype = ctypes.c_int
        L.oracle_store_copy.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, _u32p, _u32p]
        L.oracle_run_scc.restype = ctypes.c_int
        L.oracle_run_scc.argtypes = [ctypes.c_void_p, _u32p, ctypes.c_uint64, ctypes.POINTER(OracleRulePlan),
                                     ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _u64p, _u64p]
        _lib = L
    return _lib


def _p32(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def _col(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


# ---------------------------------------------------------------- generators


def splitmix64(seed: int, i: int) -> int:
    return int(lib().oracle_splitmix64(seed, i))


def er_edges(n_nodes: int, n_edges: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """The seeded ER edge set (sorted by (src, dst)), restated independently in C."""
    src = np.empty(n_edges, dtype=np.uint32)
    dst = np.empty(n_edges, dtype=np.uint32)
    got = lib().oracle_er_edges(n_nodes, n_edges, seed, _p32(src), _p32(dst))
    return src[:got].copy(), dst[:got].copy()


# ---------------------------------------------------------------- operators


def range_index(values) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """U32RangeIndex::build_slice (crates/sparkalog-storage/src/lib.rs:357-393): keys, starts, rows."""
    v = _col(values)
    n = len(v)
    keys = np.empty(max(n, 1), dtype=np.uint32)
    starts = np.empty(n + 1, dtype=np.uint32)
    rows = np.empty(max(n, 1), dtype=np.uint32)
    u = lib().oracle_range_index_build(_p32(v), n, _p32(keys), _p32(starts), _p32(rows))
    return keys[:u].copy(), starts[: u + 1].copy(), rows[:n].copy()


def join(left, right, left_key=1, right_key=0, projection=((0, 0), (1, 1)), threads=1):
    """BinaryEqualityJoin (join_cpu_serial/parallel, execution/src/lib.rs:1309-1423).

    ``left``/``right`` are (first, second) column pairs; ``projection`` is two
    (side, column) pairs with side 0 = left, 1 = right.
    """
    l0, l1 = _col(left[0]), _col(left[1])
    r0, r1 = _col(right[0]), _col(right[1])
    total = lib().oracle_join_count(_p32(l0), _p32(l1), len(l0), _p32(r0), _p32(r1), len(r0), left_key, right_key)
    o0 = np.empty(max(total, 1), dtype=np.uint32)
    o1 = np.empty(max(total, 1), dtype=np.uint32)
    (s0, c0), (s1, c1) = projection
    n = lib().oracle_join(_p32(l0), _p32(l1), len(l0), _p32(r0), _p32(r1), len(r0), left_key, right_key, s0, c0,
                          s1, c1, threads, _p32(o0), _p32(o1))
    return o0[:n].copy(), o1[:n].copy()


def distinct(rel, columns=(0, 1), threads=1):
    """BinaryDistinct (distinct_cpu_serial/parallel, execution/src/lib.rs:398-434)."""
    c0, c1 = _col(rel[0]), _col(rel[1])
    n = len(c0)
    o0 = np.empty(max(n, 1), dtype=np.uint32)
    o1 = np.empty(max(n, 1), dtype=np.uint32)
    u = lib().oracle_distinct(_p32(c0), _p32(c1), n, columns[0], columns[1], threads, _p32(o0), _p32(o1))
    return o0[:u].copy(), o1[:u].copy()


def anti_join(left, right, threads=1):
    """SortedBinaryAntiJoin (anti_join_cpu_serial/parallel, execution/src/lib.rs:672-783)."""
    l0, l1 = _col(left[0]), _col(left[1])
    r0, r1 = _col(right[0]), _col(right[1])
    o0 = np.empty(max(len(l0), 1), dtype=np.uint32)
    o1 = np.empty(max(len(l0), 1), dtype=np.uint32)
    n = lib().oracle_anti_join(_p32(l0), _p32(l1), len(l0), _p32(r0), _p32(r1), len(r0), threads, _p32(o0), _p32(o1))
    return o0[:n].copy(), o1[:n].copy()


def union(left, right, threads=1):
    """SortedBinaryUnion (union_cpu_serial/parallel, execution/src/lib.rs:934-1066)."""
    l0, l1 = _col(left[0]), _col(left[1])
    r0, r1 = _col(right[0]), _col(right[1])
    cap = max(len(l0) + len(r0), 1)
    o0 = np.empty(cap, dtype=np.uint32)
    o1 = np.empty(cap, dtype=np.uint32)
    n = lib().oracle_union(_p32(l0), _p32(l1), len(l0), _p32(r0), _p32(r1), len(r0), threads, _p32(o0), _p32(o1))
    return o0[:n].copy(), o1[:n].copy()


# ---------------------------------------------------------------- executor

ERROR_NAMES = {
    -1: "Missing", -2: "Duplicate", -3: "NotRecursive", -4: "EmptyScc", -5: "DuplicateSccRelation",
    -6: "DeltaOutsideScc", -7: "TargetOutsideScc", -8: "IncompatibleTargetPlans", -9: "MissingRuleTarget",
    -10: "IterationLimit",
}


class OracleError(RuntimeError):
    def __init__(self, code: int):
        super().__init__(ERROR_NAMES.get(code, f"error {code}"))
        self.code = code


def rule_plan(target, delta_input, right_input, left_key=1, right_key=0, projection=((0, 0), (1, 1)),
              distinct_cols=(0, 1), anti=((0, 1), (0, 1)), union_cols=((0, 1), (0, 1))) -> OracleRulePlan:
    p = OracleRulePlan()
    p.target, p.delta_input, p.right_input = target, delta_input, right_input
    p.left_key, p.right_key = left_key, right_key
    p.proj_side[0], p.proj_col[0] = projection[0]
    p.proj_side[1], p.proj_col[1] = projection[1]
    p.distinct_cols[:] = list(distinct_cols)
    p.anti_left[:] = list(anti[0])
    p.anti_right[:] = list(anti[1])
    p.union_left[:] = list(union_cols[0])
    p.union_right[:] = list(union_cols[1])
    return p


def tc_rule(path: int, edge: int) -> OracleRulePlan:
    """transitive_closure_scc (crates/sparkalog-recursion/src/generic.rs:629-661)."""
    return rule_plan(path, path, edge)


class Store:
    """RelationStore + RecursiveExecutor (crates/sparkalog-recursion/src/generic.rs:16-525)."""

    def __init__(self):
        self._h = lib().oracle_store_new()

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib is not None:
            _lib.oracle_store_free(h)

    def insert_static(self, rid: int, rel) -> None:
        c0, c1 = _col(rel[0]), _col(rel[1])
        rc = lib().oracle_store_insert_static(self._h, rid, _p32(c0), _p32(c1), len(c0))
        if rc:
            raise OracleError(rc)

    def insert_recursive(self, rid: int, full, delta) -> None:
        f0, f1, d0, d1 = _col(full[0]), _col(full[1]), _col(delta[0]), _col(delta[1])
        rc = lib().oracle_store_insert_recursive(self._h, rid, _p32(f0), _p32(f1), len(f0), _p32(d0), _p32(d1),
                                                 len(d0))
        if rc:
            raise OracleError(rc)

    def _read(self, rid: int, version: int):
        n = lib().oracle_store_len(self._h, rid, version)
        if n == (1 << 64) - 1:
            raise OracleError(-1)
        c0 = np.empty(max(n, 1), dtype=np.uint32)
        c1 = np.empty(max(n, 1), dtype=np.uint32)
        lib().oracle_store_copy(self._h, rid, version, _p32(c0), _p32(c1))
        return c0[:n].copy(), c1[:n].copy()

    def full(self, rid: int):
        return self._read(rid, 0)

    def delta(self, rid: int):
        return self._read(rid, 1)

    def run_scc(self, relations, rules, max_iterations=10_000, threads=1) -> tuple[int, int]:
        """Runs one SCC; returns (iterations, total_new_rows)."""
        rel = np.ascontiguousarray(np.asarray(relations, dtype=np.uint32))
        arr = (OracleRulePlan * max(len(rules), 1))(*rules)
        it = ctypes.c_uint64(0)
        new = ctypes.c_uint64(0)
        rc = lib().oracle_run_scc(self._h, _p32(rel), len(rel), arr, len(rules), max_iterations, threads,
                                  ctypes.byref(it), ctypes.byref(new))
        if rc:
            raise OracleError(rc)
        return int(it.value), int(new.value)

    def run_scc_bounded(self, relations, rules, rounds: int, threads=1) -> tuple[int, int, bool]:
        """Runs at most ``rounds`` rounds; returns (iterations, total_new_rows, converged)."""
        rel = np.ascontiguousarray(np.asarray(relations, dtype=np.uint32))
        arr = (OracleRulePlan * max(len(rules), 1))(*rules)
        it = ctypes.c_uint64(0)
        new = ctypes.c_uint64(0)
        rc = lib().oracle_run_scc(self._h, _p32(rel), len(rel), arr, len(rules), rounds, threads,
                                  ctypes.byref(it), ctypes.byref(new))
        if rc not in (0, -10):
            raise OracleError(rc)
        return int(it.value), int(new.value), rc == 0


def transitive_closure(src, dst, max_iterations=10_000, threads=1):
    """TC exactly as the reference's tc-fixpoint and execute_binary run it:
    EDB = sorted unique edges, FULL = DELTA = EDB, transitive_closure_scc.
    Returns ((path_first, path_second), iterations, total_new_rows)."""
    e0, e1 = btree_pairs(src, dst)
    st = Store()
    st.insert_static(0, (e0, e1))
    st.insert_recursive(1, (e0, e1), (e0, e1))
    it, new = st.run_scc([1], [tc_rule(1, 0)], max_iterations, threads)
    return st.full(1), it, new


def btree_pairs(first, second) -> tuple[np.ndarray, np.ndarray]:
    """The BTreeSet<[u32; 2]> order execute_binary builds (subset.rs:381-398): sorted, unique."""
    packed = (np.asarray(first, dtype=np.uint64) << np.uint64(32)) | np.asarray(second, dtype=np.uint64)
    packed = np.unique(packed)
    return (packed >> np.uint64(32)).astype(np.uint32), (packed & np.uint64(0xFFFFFFFF)).astype(np.uint32)


# ---------------------------------------------------------------- execute_binary


@dataclass
class SeedPlan:
    """BinarySeedPlan (subset.rs:18-23)."""

    target: int
    source: int
    columns: tuple[int, int]


@dataclass
class SccPlan:
    relations: list[int]
    rules: list[OracleRulePlan]
    seeds: list[SeedPlan] = field(default_factory=list)


def execute_binary(predicate_count: int, facts: list[tuple[int, tuple[int, int]]], sccs: list[SccPlan],
                   max_iterations: int = 10_000, threads: int = 1):
    """execute_binary (crates/sparkalog-datalog/src/subset.rs:369-414).

    Facts go into one sorted set per relation; each SCC's seed clauses project
    their source's *current set* (facts and earlier seeds, not derived rows)
    into the target; every relation then enters the store, recursive ones with
    FULL = DELTA; the SCCs run in order. Returns (store, [(iterations, new_rows)]).
    """
    rows: list[set] = [set() for _ in range(predicate_count)]
    for rel, tup in facts:
        rows[rel].add((int(tup[0]), int(tup[1])))
    for scc in sccs:
        for seed in scc.seeds:
            for tup in sorted(rows[seed.source]):
                rows[seed.target].add((tup[seed.columns[0]], tup[seed.columns[1]]))
    recursive = {r for scc in sccs for r in scc.relations}
    st = Store()
    for rid, tuples in enumerate(rows):
        ordered = sorted(tuples)
        c0 = np.array([t[0] for t in ordered], dtype=np.uint32)
        c1 = np.array([t[1] for t in ordered], dtype=np.uint32)
        if rid in recursive:
            st.insert_recursive(rid, (c0, c1), (c0, c1))
        else:
            st.insert_static(rid, (c0, c1))
    summaries = [st.run_scc(scc.relations, scc.rules, max_iterations, threads) for scc in sccs]
    return st, summaries


# ---------------------------------------------------------------- GeneralCpu (small inputs)


@dataclass
class Atom:
    """PlannedAtom (relational/src/lib.rs:104-109): terms are ("b", id) bindings or ("v", value) constants."""

    relation: int
    terms: list[tuple[str, int]]
    delta: bool = False


@dataclass
class Clause:
    """RelationalClausePlan (relational/src/lib.rs:113-121)."""

    target: int
    head: list[tuple[str, int]]
    positive: list[Atom]
    negative: list[Atom] = field(default_factory=list)


@dataclass
class GeneralScc:
    relations: list[int]
    recursive: bool
    seeds: list[Clause]
    recursive_variants: list[Clause]


def _match(binding: list, terms, tup) -> bool:
    # match_atom, general.rs:553-573
    for (kind, x), value in zip(terms, tup):
        if kind == "v":
            if x != value:
                return False
        else:
            cur = binding[x]
            if cur is None:
                binding[x] = value
            elif cur != value:
                return False
    return True


def _evaluate_clause(clause: Clause, full: dict, delta: dict) -> set:
    # evaluate_clause, general.rs:478-551 (nested-loop joins, negation as a
    # scan of the negated relation's FULL). Join order and liveness pruning
    # (optimize_general) change only cost, not the result set.
    ids = [x for kind, x in clause.head if kind == "b"]
    for atom in clause.positive + clause.negative:
        ids += [x for kind, x in atom.terms if kind == "b"]
    width = max(ids) + 1 if ids else 0
    bindings = [[None] * width]
    for atom in clause.positive:
        rows = delta[atom.relation] if atom.delta else full[atom.relation]
        joined = []
        for b in bindings:
            for tup in sorted(rows):
                if len(tup) != len(atom.terms):
                    continue
                cand = list(b)
                if _match(cand, atom.terms, tup):
                    joined.append(cand)
        bindings = joined
        if not bindings:
            break
    for atom in clause.negative:
        rows = full[atom.relation]
        bindings = [b for b in bindings
                    if not any(len(t) == len(atom.terms) and _match(list(b), atom.terms, t) for t in rows)]
        if not bindings:
            break
    out = set()
    for b in bindings:
        out.add(tuple(b[x] if kind == "b" else x for kind, x in clause.head))
    return out


def general_cpu(predicate_count: int, facts, strata: list[list[GeneralScc]], max_iterations: int = 10_000):
    """execute_general / execute_scc (general.rs:371-443).

    Returns (full, summaries) with full[relation] a set of tuples and one
    (relations_rows, iterations, new_rows) summary per SCC, non-recursive SCCs
    included (iterations 1 if they have seeds, else 0).
    """
    full = {r: set() for r in range(predicate_count)}
    delta = {r: set() for r in range(predicate_count)}
    for rel, tup in facts:
        full[rel].add(tuple(int(x) for x in tup))
    summaries = []
    for stratum in strata:
        for scc in stratum:
            contributions = {}
            for clause in scc.seeds:
                contributions.setdefault(clause.target, set()).update(_evaluate_clause(clause, full, delta))
            for target, tuples in contributions.items():
                full[target] |= tuples
            if not scc.recursive:
                summaries.append(([(r, len(full[r])) for r in scc.relations], 1 if scc.seeds else 0, 0))
                continue
            for r in scc.relations:
                delta[r] = set(full[r])
            iterations = 0
            total_new = 0
            while any(delta[r] for r in scc.relations):
                if iterations >= max_iterations:
                    raise OracleError(-10)
                contributions = {}
                for clause in scc.recursive_variants:
                    contributions.setdefault(clause.target, set()).update(_evaluate_clause(clause, full, delta))
                nxt = {r: set() for r in scc.relations}
                for target, tuples in contributions.items():
                    nxt[target] |= {t for t in tuples if t not in full[target]}
                for r in scc.relations:
                    total_new += len(nxt[r])
                    full[r] |= nxt[r]
                    delta[r] = nxt[r]
                iterations += 1
            summaries.append(([(r, len(full[r])) for r in scc.relations], iterations, total_new))
    return full, summaries


# ---------------------------------------------------------------- reference CUDA


def reference_cuda() -> ctypes.CDLL | None:
    """The reference's column_ops.cu built unmodified for sm_100a, if it was built."""
    if not REF_CUDA_PATH.exists():
        return None
    return ctypes.CDLL(str(REF_CUDA_PATH))


# ---------------------------------------------------------------------------
# Filter (crates/sparkalog-execution/src/lib.rs:1681-1760): ascending row ids
# whose value satisfies the predicate; operation codes 0 ==, 1 !=, 2 <, 3 <=,
# 4 >, 5 >= (crates/sparkalog-relational/src/lib.rs:144-164).
# ---------------------------------------------------------------------------
def _filter_matches(value: int, op: int, operand: int) -> bool:
    return {0: value == operand, 1: value != operand, 2: value < operand, 3: value <= operand,
            4: value > operand, 5: value >= operand}.get(op, False)


def filter_serial(values, op: int, operand: int) -> np.ndarray:
    """filter_cpu_serial (lib.rs:1681-1702): one pass, row ids in order."""
    return np.array([row for row, v in enumerate(np.asarray(values).tolist()) if _filter_matches(v, op, operand)],
                    dtype=np.uint32)


def filter_parallel(values, op: int, operand: int, workers: int = 8) -> np.ndarray:
    """filter_cpu_parallel (lib.rs:1705-1760): per-chunk flags, an exclusive scan
    of the chunk counts, ids written at the chunk offsets."""
    v = np.asarray(values, dtype=np.uint32)
    n = len(v)
    if n == 0:
        return np.zeros(0, dtype=np.uint32)
    chunk = -(-n // min(workers, n))
    cmp = {0: np.equal, 1: np.not_equal, 2: np.less, 3: np.less_equal, 4: np.greater, 5: np.greater_equal}
    flags = [cmp[op](v[i:i + chunk], np.uint32(operand)) if op in cmp else np.zeros(len(v[i:i + chunk]), bool)
             for i in range(0, n, chunk)]
    counts = [int(f.sum()) for f in flags]
    out = np.zeros(sum(counts), dtype=np.uint32)
    off = 0
    for c, (i, f) in enumerate(zip(range(0, n, chunk), flags)):
        out[off:off + counts[c]] = np.nonzero(f)[0].astype(np.uint32) + np.uint32(i)
        off += counts[c]
    return out


# ---------------------------------------------------------------------------
# load_binary_u32 (crates/sparkalog-storage/src/io.rs:72-138): count_rows
# first (a Git LFS pointer header anywhere is an error), then populate_columns
# line by line: trim, skip empty / '#' / '%' lines, exactly two whitespace
# separated fields, each parsed as u32 (optional '+', decimal digits).
# ---------------------------------------------------------------------------
class OracleLoadError(Exception):
    def __init__(self, kind: str, line: int = 0, column: int = 0, value: str | None = None):
        super().__init__(kind, line, column, value)
        self.kind, self.line, self.column, self.value = kind, line, column, value


_LFS = "version https://git-lfs.github.com/spec/v1"
_ASCII_SPACE = " \t\n\x0b\x0c\r"


def _parse_u32(field: str) -> int | None:
    digits = field[1:] if field.startswith("+") else field
    if not digits or any(c not in "0123456789" for c in digits):
        return None
    v = int(digits)
    return v if v <= 0xFFFFFFFF else None


def load_binary_u32(data: bytes) -> tuple[np.ndarray, np.ndarray]:
    lines = data.decode().split("\n")
    if lines and lines[-1] == "":
        lines.pop()  # str::lines(): a final '\n' ends the last line
    for line in lines:  # count_rows
        t = line.strip(_ASCII_SPACE)
        if t and t[0] not in "#%" and t == _LFS:
            raise OracleLoadError("GitLfsPointer")
    first, second = [], []
    for index, line in enumerate(lines):  # populate_columns
        t = line.strip(_ASCII_SPACE)
        if not t or t[0] in "#%":
            continue
        fields = [f for f in t.replace("\t", " ").replace("\x0b", " ").replace("\x0c", " ").replace("\r", " ")
                  .split(" ") if f]
        if len(fields) != 2:
            raise OracleLoadError("InvalidFieldCount", index + 1)
        for column, f in enumerate(fields, start=1):
            v = _parse_u32(f)
            if v is None:
                raise OracleLoadError("InvalidU32", index + 1, column, f)
            (first if column == 1 else second).append(v)
    return np.array(first, dtype=np.uint32), np.array(second, dtype=np.uint32)


def intern(values, catalog: dict | None = None) -> tuple[np.ndarray, dict]:
    """ValueCatalog::intern (crates/sparkalog-datalog/src/catalog.rs:108-117) applied to
    each value in order: an unseen value gets id len(catalog)."""
    catalog = {} if catalog is None else catalog
    out = np.empty(len(values), dtype=np.uint32)
    for i, v in enumerate(np.asarray(values, dtype=np.uint32).tolist()):
        if v not in catalog:
            catalog[v] = len(catalog)
        out[i] = catalog[v]
    return out, catalog


# ---------------------------------------------------------------------------
# load_delimited (crates/sparkalog-datalog/src/database.rs:165-177) over
# parse_delimited_parallel (crates/sparkalog-datalog/src/ingest.rs:20-120):
# str::lines (split at '\n', a '\r' before it dropped, no piece after a
# final '\n'), the header line skipped, lines that trim to nothing dropped,
# then each record split at the delimiter byte: a field starting with '"' is
# a quoted String ('""' is a quote) that must be followed by the delimiter or
# the end; any other field is trimmed and is a U32 when it parses as one,
# else a Symbol. Errors carry the 1-based line and byte column. Values are
# then interned row by row (ValueCatalog, catalog.rs:98-127), String, Symbol
# and U32 being distinct keys.
# ---------------------------------------------------------------------------
class OracleDelimitedError(Exception):
    def __init__(self, line: int, column: int, message: str):
        super().__init__(line, column, message)
        self.line, self.column, self.message = line, column, message


class OracleArityError(Exception):
    """DatabaseError::Arity (database.rs:98-104): a row with the wrong number of values."""

    def __init__(self, expected: int, actual: int):
        super().__init__(expected, actual)
        self.expected, self.actual = expected, actual


# char::is_whitespace (the Unicode White_Space property), used by str::trim.
_RUST_WHITESPACE = set("\t\n\x0b\x0c\r \x85\xa0\u1680\u2028\u2029\u202f\u205f\u3000") | {
    chr(c) for c in range(0x2000, 0x200B)}


def _rust_trim(s: str) -> str:
    a, b = 0, len(s)
    while a < b and s[a] in _RUST_WHITESPACE:
        a += 1
    while b > a and s[b - 1] in _RUST_WHITESPACE:
        b -= 1
    return s[a:b]


def _rust_lines(text: str) -> list[str]:
    # A '\r' is dropped only before a '\n' (str::lines strips "\n", then "\r").
    pieces = text.split("\n")
    out = [p[:-1] if p.endswith("\r") else p for p in pieces[:-1]]
    if pieces[-1]:
        out.append(pieces[-1])
    return out


def _utf8_len(lead: int) -> int:
    return 1 if lead < 0x80 else 2 if lead < 0xE0 else 3 if lead < 0xF0 else 4


def _parse_record(record: str, line: int, delimiter: int) -> list[tuple]:
    b = record.encode()
    n, pos, fields = len(b), 0, []
    while True:
        column = pos + 1
        if pos < n and b[pos] == 0x22:
            pos += 1
            value, closed = bytearray(), False
            while pos < n:
                if b[pos] == 0x22:
                    if pos + 1 < n and b[pos + 1] == 0x22:
                        value += b'"'
                        pos += 2
                    else:
                        pos += 1
                        closed = True
                        break
                else:
                    step = _utf8_len(b[pos])
                    value += b[pos:pos + step]
                    pos += step
            if not closed:
                raise OracleDelimitedError(line, column, "unterminated quoted field")
            fields.append(("string", value.decode()))
            if pos < n and b[pos] != delimiter:
                raise OracleDelimitedError(line, pos + 1, "expected delimiter after quoted field")
        else:
            start = pos
            while pos < n and b[pos] != delimiter:
                pos += 1
            value = _rust_trim(b[start:pos].decode())
            if not value:
                raise OracleDelimitedError(line, column, "empty fields are not values")
            number = _parse_u32(value)
            fields.append(("u32", number) if number is not None else ("symbol", value))
        if pos == n:
            break
        pos += 1
        if pos == n:
            raise OracleDelimitedError(line, pos, "record ends with an empty field")
    return fields


def parse_delimited(source: str, delimiter: str = ",", has_header: bool = False) -> list[list[tuple]]:
    """parse_delimited_parallel (ingest.rs:20-41): rows of ("u32", n) /
    ("string", s) / ("symbol", s) values in input order."""
    d = ord(delimiter)
    if chr(d) in " \t\n\x0c\r" and chr(d) != "\t":
        raise OracleDelimitedError(0, 0, "delimiter must be a visible ASCII byte or tab")
    rows = []
    for index, record in enumerate(_rust_lines(source)):
        if has_header and index == 0:
            continue
        if not _rust_trim(record):
            continue
        rows.append(_parse_record(record, index + 1, d))
    return rows


def load_delimited(source: str, arity: int, delimiter: str = ",", has_header: bool = False,
                   catalog: dict | None = None) -> tuple[np.ndarray, dict]:
    """Database::load_delimited (database.rs:165-177): every row must have
    `arity` values (Database::insert, :80-110); values are interned in row
    order. Returns the rows as value ids, shape (rows, arity), and the catalog."""
    catalog = {} if catalog is None else catalog
    rows = parse_delimited(source, delimiter, has_header)
    out = np.empty((len(rows), arity), dtype=np.uint32)
    for r, row in enumerate(rows):
        if len(row) != arity:
            raise OracleArityError(arity, len(row))
        for c, value in enumerate(row):
            if value not in catalog:
                catalog[value] = len(catalog)
            out[r, c] = catalog[value]
    return out, catalog


def general_tc_c(src, dst, max_rounds: int = 10_000, time_cap_s: float = 1e30) -> dict:
    """GeneralCpu's nested-loop evaluation of transitive closure (oracle.cpp,
    general.rs:393-536), bounded by rounds and a time cap: completed rounds,
    their new tuples, the tuple tests made, seconds, and whether it converged."""
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    rounds, new, tests = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_uint64(0)
    seconds, converged = ctypes.c_double(0.0), ctypes.c_int(0)
    lib().oracle_general_tc(_p32(s), _p32(d), len(s), max_rounds, time_cap_s, ctypes.byref(rounds),
                            ctypes.byref(new), ctypes.byref(tests), ctypes.byref(seconds), ctypes.byref(converged))
    return {"rounds": rounds.value, "new_rows": new.value, "tests": tests.value, "seconds": seconds.value,
            "converged": bool(converged.value)}


def load_binary_u32_c(data: bytes) -> tuple[np.ndarray, np.ndarray]:
    """The C restatement of load_binary_u32 (oracle.cpp), for large texts and timing."""
    cap = data.count(b"\n") + 1
    first = np.empty(cap, dtype=np.uint32)
    second = np.empty(cap, dtype=np.uint32)
    rows, line, column = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_int(0)
    rc = lib().oracle_load_binary_u32(data, len(data), _p32(first), _p32(second), cap, ctypes.byref(rows),
                                      ctypes.byref(line), ctypes.byref(column))
    if rc:
        raise OracleLoadError({1: "GitLfsPointer", 2: "InvalidFieldCount", 3: "InvalidU32"}[rc], int(line.value),
                              int(column.value) if rc == 3 else 0)
    return first[:rows.value].copy(), second[:rows.value].copy()


def intern_c(values) -> np.ndarray:
    """The C restatement of ValueCatalog::intern over one batch (oracle.cpp)."""
    v = np.ascontiguousarray(np.asarray(values, dtype=np.uint32))
    out = np.empty_like(v)
    lib().oracle_intern_u32(_p32(v), len(v), _p32(out))
    return out
