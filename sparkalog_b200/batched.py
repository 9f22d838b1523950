"""Batched fixpoints: thousands of independent transitive closures in one run.

Each instance's node ids are tagged with its instance number in the high bits
of both columns (``instance << id_bits | local_id``). The tagged instances
form one disjoint union, so a single device fixpoint computes every
instance's closure at once: the radix sort, the join and the merges all sort
by the instance prefix first, i.e. they run segmented by instance inside the
same persistent kernels, and a round's launches are shared by every instance
that is still active. The engine's per-segment activity tracking gives each
instance the iteration count its own RecursiveExecutor::run would report
(crates/sparkalog-recursion/src/generic.rs:472-516), and the union's FULL
splits back into per-instance results.

With 14-bit local ids the 12 remaining bits tag up to 4,096 instances.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .recursion import RecursiveExecutor, RelationStore, transitive_closure_scc
from .relational import RelationId


@dataclass
class InstanceResult:
    path: tuple[np.ndarray, np.ndarray]
    iterations: int
    new_rows: int


def _btree(src, dst) -> tuple[np.ndarray, np.ndarray]:
    """Sorted, deduplicated pairs (the BTreeSet execute_binary builds)."""
    packed = np.unique((np.asarray(src, dtype=np.uint64) << np.uint64(32)) | np.asarray(dst, dtype=np.uint64))
    return (packed >> np.uint64(32)).astype(np.uint32), (packed & np.uint64(0xFFFFFFFF)).astype(np.uint32)


class BatchedTransitiveClosure:
    """Runs the TC program over many independent edge sets in one device fixpoint."""

    def __init__(self, instances: list[tuple[np.ndarray, np.ndarray]], id_bits: int = 14, stream=None):
        if not 1 <= id_bits <= 31:
            raise ValueError("id_bits must be in [1, 31]")
        if len(instances) > (1 << (32 - id_bits)):
            raise ValueError(f"at most {1 << (32 - id_bits)} instances with {id_bits}-bit ids")
        self.id_bits = id_bits
        self.stream = stream
        self.edges = [_btree(s, d) for s, d in instances]
        limit = 1 << id_bits
        for k, (s, d) in enumerate(self.edges):
            if len(s) and (int(s.max()) >= limit or int(d.max()) >= limit):
                raise ValueError(f"instance {k} has node ids >= 2^{id_bits}")

    def tagged_edges(self) -> tuple[np.ndarray, np.ndarray]:
        """The union's EDB: instance-major, so it is sorted when every instance is."""
        firsts, seconds = [], []
        for k, (s, d) in enumerate(self.edges):
            tag = np.uint32(k << self.id_bits)
            firsts.append(s | tag)
            seconds.append(d | tag)
        if not firsts:
            return np.zeros(0, dtype=np.uint32), np.zeros(0, dtype=np.uint32)
        return np.concatenate(firsts), np.concatenate(seconds)

    def run(self, max_iterations: int = 10_000, edges=None) -> tuple[list[InstanceResult], object]:
        """One fixpoint over the union; returns per-instance results and the run's SccSummary.

        ``edges`` may pass the tagged EDB already resident on the device
        (a pair of int32 CUDA tensors) to skip the upload."""
        first, second = edges if edges is not None else self.tagged_edges()
        store = RelationStore(self.stream)
        store.insert_static(0, (first, second))
        store.insert_recursive(1, (first, second), (first, second))
        executor = RecursiveExecutor.compile(transitive_closure_scc(RelationId(1), RelationId(0)), store)
        executor.track_segments(self.id_bits, len(self.edges))
        summary = executor.run(store, max_iterations)
        seen, new_rows = executor.segment_stats()
        executor.close()
        f0, f1 = store.full(1)
        store.close()
        return self.split(f0, f1, seen, new_rows), summary

    def split(self, f0, f1, seen, new_rows) -> list[InstanceResult]:
        mask = np.uint32((1 << self.id_bits) - 1)
        tags = f0 >> np.uint32(self.id_bits)
        bounds = np.searchsorted(tags, np.arange(len(self.edges) + 1, dtype=np.uint32), side="left")
        out = []
        for k in range(len(self.edges)):
            a, b = bounds[k], bounds[k + 1]
            iterations = int(seen[k]) + 1 if len(self.edges[k][0]) else 0
            out.append(InstanceResult((f0[a:b] & mask, f1[a:b] & mask), iterations, int(new_rows[k])))
        return out

    def run_serial(self, max_iterations: int = 10_000) -> list[InstanceResult]:
        """The same instances one at a time through the same engine (the batching baseline)."""
        out = []
        for s, d in self.edges:
            store = RelationStore(self.stream)
            store.insert_static(0, (s, d))
            store.insert_recursive(1, (s, d), (s, d))
            executor = RecursiveExecutor.compile(transitive_closure_scc(RelationId(1), RelationId(0)), store)
            summary = executor.run(store, max_iterations)
            executor.close()
            path = store.full(1)
            store.close()
            out.append(InstanceResult(path, summary.iterations, summary.total_new_rows))
        return out
