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
        store, summary, seen, new_rows = self.run_device(max_iterations, edges)
        try:
            return self.collect(store, seen, new_rows), summary
        finally:
            store.close()

    def run_device(self, max_iterations: int = 10_000, edges=None):
        """The device part of run(): the fixpoint, leaving the union's FULL in the
        returned store (the caller closes it); also returns the SccSummary and the
        per-instance (last active round, new rows)."""
        first, second = edges if edges is not None else self.tagged_edges()
        store = RelationStore(self.stream)
        store.insert_static(0, (first, second))
        store.insert_recursive(1, (first, second), (first, second))
        executor = RecursiveExecutor.compile(transitive_closure_scc(RelationId(1), RelationId(0)), store)
        executor.track_segments(self.id_bits, len(self.edges))
        summary = executor.run(store, max_iterations)
        seen, new_rows = executor.segment_stats()
        executor.close()
        return store, summary, seen, new_rows

    def collect(self, store: RelationStore, seen, new_rows) -> list[InstanceResult]:
        """Per-instance results from the union's FULL: the instance tags are cleared on the
        device, the columns come back once, and each instance is a slice of them (its
        FULL holds its seed plus its new rows, and instances are contiguous)."""
        import torch

        n = store.rows(1)
        d0 = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
        d1 = torch.empty_like(d0)
        store.read_into(1, 0, d0, d1)
        mask = (1 << self.id_bits) - 1
        h0 = torch.empty(max(n, 1), dtype=torch.int32, pin_memory=True)
        h1 = torch.empty_like(h0, pin_memory=True)
        h0.copy_(torch.bitwise_and(d0, mask), non_blocking=True)
        h1.copy_(torch.bitwise_and(d1, mask), non_blocking=True)
        torch.cuda.synchronize()
        return self._slices(h0.numpy()[:n].view(np.uint32), h1.numpy()[:n].view(np.uint32), seen, new_rows)

    def split(self, f0, f1, seen, new_rows) -> list[InstanceResult]:
        """Per-instance results from the union's FULL read to the host with its tags."""
        mask = np.uint32((1 << self.id_bits) - 1)
        return self._slices(np.asarray(f0, dtype=np.uint32) & mask, np.asarray(f1, dtype=np.uint32) & mask, seen,
                            new_rows)

    def _slices(self, f0, f1, seen, new_rows) -> list[InstanceResult]:
        n = len(f0)
        sizes = np.array([len(e[0]) for e in self.edges], dtype=np.int64) + np.asarray(new_rows, dtype=np.int64)
        bounds = np.concatenate([[0], np.cumsum(sizes)])
        if bounds[-1] != n:
            raise RuntimeError(f"per-instance sizes sum to {bounds[-1]}, FULL holds {n} rows")
        out = []
        for k in range(len(self.edges)):
            a, b = bounds[k], bounds[k + 1]
            iterations = int(seen[k]) + 1 if len(self.edges[k][0]) else 0
            out.append(InstanceResult((f0[a:b], f1[a:b]), iterations, int(new_rows[k])))
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
