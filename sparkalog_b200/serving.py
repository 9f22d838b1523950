"""Serving: continuous batching of transitive-closure requests on one GPU.

Each request is the TC program over its own edge set. The server keeps one
device-resident store: relation 0 is the union of every admitted request's
EDB, relation 1 the union of their path relations, each request's rows tagged
with a slot number in the high bits of both columns (node ids keep the low
``id_bits``). One shared RecursiveExecutor advances every active request by a
round at a time, so the iterations of concurrent requests run in the same
kernel launches. Between rounds the server

* admits requests that have arrived, while a slot is free and the HBM budget
  (estimated from each request's edge count times the FULL/EDB growth seen in
  earlier requests) allows: their tagged edges are appended to the EDB and,
  as seed, to FULL and DELTA of the path relation, which starts their
  fixpoints (crates/sparkalog-datalog/src/subset.rs:381-408 seeds path with
  the edges the same way);
* completes every request that derived no new rows in the last round: its
  DELTA is empty, so its fixpoint is done. Its FULL slice is copied out and
  its slot is retired; retired slots' rows are purged from the store in one
  pass when free slots run out or the budget needs the room.

Per request, the result (rows and iteration count) equals the request run
alone: tags keep requests disjoint, and the executor's per-segment activity
gives each one the number of rounds its own RecursiveExecutor::run would take.

A step may run several rounds (``rounds_per_step``); the executor then runs
the small ones as one device-driven graph launch. Results can be completed
into device memory (``readout="device"``: each completion holds two CUDA
tensors) or read to the host. ``LanedServer`` splits requests by size into
lanes, each with its own CUDA stream (the lane of small requests at a higher
stream priority) and its own host thread: small requests are batched in a
FixpointServer, large ones run one at a time beside them (SequentialLane), so
a small request does not wait behind the long rounds of a large one.
"""

from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .recursion import RecursiveExecutor, RelationStore, transitive_closure_scc
from .relational import RelationId

EDB, PATH = 0, 1


@dataclass
class ServeRequest:
    request_id: int
    arrival_s: float
    src: np.ndarray
    dst: np.ndarray


@dataclass
class Completion:
    request_id: int
    path: tuple[np.ndarray, np.ndarray]
    iterations: int
    new_rows: int
    arrival_s: float
    admitted_s: float
    finished_s: float

    @property
    def latency_s(self) -> float:
        return self.finished_s - self.arrival_s


@dataclass
class _Active:
    request: ServeRequest
    slot: int
    admit_round: int
    admitted_s: float
    base_new_rows: int
    est_bytes: float


class FixpointServer:
    """Continuous-batching TC server over one device-resident store."""

    def __init__(self, id_bits: int = 23, budget_bytes: float = 120e9, growth_prior: float = 16.0, stream=None,
                 clock=time.perf_counter, readout: str = "host", rounds_per_step: int = 1):
        if readout not in ("host", "device"):
            raise ValueError("readout is 'host' or 'device'")
        self.shift = id_bits
        self.slots = 1 << (32 - id_bits)
        self.budget = budget_bytes
        self.growth = growth_prior
        self.clock = clock
        self.readout = readout
        self.rounds_per_step = max(1, int(rounds_per_step))
        self.store = RelationStore(stream)
        empty = (np.zeros(0, dtype=np.uint32), np.zeros(0, dtype=np.uint32))
        self.store.insert_static(EDB, empty)
        self.store.insert_recursive(PATH, empty, empty)
        self.executor = RecursiveExecutor.compile(transitive_closure_scc(RelationId(PATH), RelationId(EDB)),
                                                  self.store)
        self.executor.track_segments(self.shift, self.slots)
        self.free = list(range(self.slots - 1, -1, -1))
        self.retired: list[int] = []
        self.retired_bytes = 0.0
        self.active: dict[int, _Active] = {}
        self.rounds = 0
        self._stage: tuple = ()  # (page-locked tensors, their u32 views)
        self.completions: list[Completion] = []

    # ------------------------------------------------------------ admission

    def estimate_bytes(self, edges: int) -> float:
        """HBM estimate of one request: EDB + FULL rows (8 B packed) with the
        growth factor observed so far, doubled for merge and sort buffers."""
        return 16.0 * edges * (1.0 + self.growth)

    def resident_bytes(self) -> float:
        return sum(a.est_bytes for a in self.active.values()) + self.retired_bytes

    def can_admit(self, request: ServeRequest, batch: list[ServeRequest] = ()) -> bool:
        """Whether `request` fits next to the active requests and the `batch`
        already chosen for admission (a free slot each, and the HBM budget)."""
        if len(self.free) <= len(batch) and self.retired:
            self.purge()
        if len(self.free) <= len(batch):
            return False
        reserved = sum(self.estimate_bytes(len(r.src)) for r in batch)
        need = self.estimate_bytes(len(request.src))
        if self.resident_bytes() + reserved + need > self.budget and self.retired:
            self.purge()
        return self.resident_bytes() + reserved + need <= self.budget or (not self.active and not batch)

    def _staging(self, rows: int) -> tuple[np.ndarray, np.ndarray]:
        """Two page-locked u32 columns of at least `rows` entries, kept across
        admissions: tagged edges are written there once and copied to the
        device at full link speed."""
        if not self._stage or len(self._stage[1][0]) < rows:
            cap = max(rows, 2 * len(self._stage[1][0]) if self._stage else 1 << 20)
            pin = torch.cuda.is_available()
            t = [torch.empty(cap, dtype=torch.int32, pin_memory=pin) for _ in range(2)]
            self._stage = (t, [x.numpy().view(np.uint32) for x in t])
        return self._stage[1][0], self._stage[1][1]

    def admit(self, requests: list[ServeRequest]) -> None:
        """Appends the requests' tagged edges to the EDB and, as seed, to FULL/DELTA of path."""
        if not requests:
            return
        now = self.clock()
        _, new_rows = self.executor.segment_stats()
        cols = [(np.asarray(r.src, dtype=np.uint32), np.asarray(r.dst, dtype=np.uint32)) for r in requests]
        first, second = self._staging(sum(len(s) for s, _ in cols))
        off = 0
        for req, (s, d) in zip(requests, cols):
            if len(s) != len(d):
                raise ValueError(f"request {req.request_id} has columns of different lengths")
            if len(s) and max(int(s.max()), int(d.max())) >= (1 << self.shift):
                raise ValueError(f"request {req.request_id} has node ids >= 2^{self.shift}")
            slot = self.free.pop()
            if len(s) == 0:
                # No seed: the fixpoint runs zero rounds.
                self.completions.append(Completion(req.request_id, (s, d), 0, 0, req.arrival_s, now, now))
                self.free.append(slot)
                continue
            # Raw edge lists, tagged in the staging columns: the device append
            # sorts and deduplicates them.
            tag = np.uint32(slot << self.shift)
            np.bitwise_or(s, tag, out=first[off:off + len(s)])
            np.bitwise_or(d, tag, out=second[off:off + len(s)])
            off += len(s)
            self.active[slot] = _Active(req, slot, self.rounds, now, int(new_rows[slot]),
                                        self.estimate_bytes(len(s)))
        if off:
            # Each append has finished reading the staging columns when it returns.
            self.store.append(EDB, (first[:off], second[:off]))
            self.store.append(PATH, (first[:off], second[:off]))

    # ------------------------------------------------------------ rounds

    def step(self) -> list[Completion]:
        """Up to rounds_per_step rounds for every active request, then completes
        the finished ones."""
        if not self.active:
            return []
        summary, _ = self.executor.step(self.store, self.rounds_per_step)
        self.rounds += summary.iterations
        seen, new_rows = self.executor.segment_stats()
        done = [slot for slot in self.active if int(seen[slot]) != self.rounds]
        finished = []
        now = None
        for slot in done:
            a = self.active.pop(slot)
            f0, f1 = self.store.extract_segment(PATH, self.shift, slot, untag=True, device=self.readout == "device")
            iterations = int(seen[slot]) - a.admit_round + 1 if int(seen[slot]) > a.admit_round else 1
            now = self.clock()
            c = Completion(a.request.request_id, (f0, f1), iterations,
                           int(new_rows[slot]) - a.base_new_rows, a.request.arrival_s, a.admitted_s, now)
            finished.append(c)
            edges = max(len(a.request.src), 1)
            self.growth = 0.8 * self.growth + 0.2 * (len(f0) / edges)
            self.retired.append(slot)
            self.retired_bytes += 16.0 * (len(f0) + edges)
        self.completions.extend(finished)
        # Retired rows cost every later round (FULL holds them): drop them at
        # once when the server falls idle or they outweigh the live rows.
        if self.retired and (not self.active or self.retired_bytes > self.resident_bytes() - self.retired_bytes):
            self.purge()
        return finished

    def purge(self) -> None:
        """Removes every retired request's rows from the store and frees its slot."""
        if not self.retired:
            return
        self.store.remove_segments(EDB, self.shift, self.retired)
        self.store.remove_segments(PATH, self.shift, self.retired)
        self.free.extend(self.retired)
        self.retired = []
        self.retired_bytes = 0.0

    def close(self) -> None:
        self.executor.close()
        self.store.close()


@dataclass
class ServeReport:
    completions: list[Completion] = field(default_factory=list)
    wall_s: float = 0.0
    rounds: int = 0

    def latencies(self) -> np.ndarray:
        return np.array([c.latency_s for c in self.completions])

    def summary(self) -> dict:
        lat = self.latencies()
        tuples = sum(c.new_rows for c in self.completions)
        return {"requests": len(self.completions), "wall_s": self.wall_s,
                "p50_ms": float(np.percentile(lat, 50) * 1e3) if len(lat) else None,
                "p99_ms": float(np.percentile(lat, 99) * 1e3) if len(lat) else None,
                "requests_per_s": len(self.completions) / self.wall_s if self.wall_s else None,
                "derived_tuples_per_s": tuples / self.wall_s if self.wall_s else None,
                "rounds": self.rounds}


def serve(requests: list[ServeRequest], server: FixpointServer, realtime: bool = True) -> ServeReport:
    """Replays an arrival stream against the continuous-batching server."""
    pending = sorted(requests, key=lambda r: r.arrival_s)
    start = server.clock()
    server.clock = (lambda base=server.clock: base() - start)
    i = 0
    while i < len(pending) or server.active:
        now = server.clock()
        batch = []
        while i < len(pending) and (pending[i].arrival_s <= now or not realtime):
            if not server.can_admit(pending[i], batch):
                break
            batch.append(pending[i])
            i += 1
        server.admit(batch)
        if server.active:
            server.step()
        elif i < len(pending):
            wait = pending[i].arrival_s - server.clock()
            if wait > 0:
                time.sleep(wait)
    report = ServeReport(list(server.completions), server.clock(), server.rounds)
    return report


class SequentialLane:
    """A lane that runs its requests one after another, each alone through the
    engine (a fresh store and executor, as serve_one_at_a_time does), with
    the FixpointServer interface that serve_laned drives. For large requests:
    their rounds already fill the GPU, so sharing rounds with others gains
    nothing, while every admission into a shared store re-merges and
    re-indexes everything resident (which made batched large requests three
    times slower than running them alone)."""

    def __init__(self, stream=None, clock=time.perf_counter, readout: str = "host"):
        if readout not in ("host", "device"):
            raise ValueError("readout is 'host' or 'device'")
        self.stream = stream
        self.clock = clock
        self.readout = readout
        self.active: dict[int, ServeRequest] = {}
        self.completions: list[Completion] = []
        self.rounds = 0
        self._admitted = 0.0

    def can_admit(self, request: ServeRequest, batch: list[ServeRequest] = ()) -> bool:
        return not self.active and not batch

    def admit(self, requests: list[ServeRequest]) -> None:
        for r in requests:
            self.active[r.request_id] = r
            self._admitted = self.clock()

    def step(self) -> list[Completion]:
        finished = []
        for rid, req in list(self.active.items()):
            path, iterations, new_rows = _run_alone(req, self.stream, self.readout)
            self.rounds += iterations
            c = Completion(rid, path, iterations, new_rows, req.arrival_s, self._admitted, self.clock())
            finished.append(c)
            del self.active[rid]
        self.completions.extend(finished)
        return finished

    def close(self) -> None:
        pass


class LanedServer:
    """Requests split by edge count into lanes (lane k takes requests with at
    most bounds[k] edges, the last lane the rest), each lane stepped by its
    own host thread on its own stream. The lanes of smaller requests are
    FixpointServers (continuous batching in one store); the last lane runs
    its large requests one at a time (SequentialLane) unless
    ``batch_last=True``. Lane 0 (the smallest requests) runs at the highest
    stream priority."""

    def __init__(self, bounds=(1 << 17,), budget_bytes: float = 120e9, shares=None, readout: str = "host",
                 rounds_per_step: int = 1, clock=time.perf_counter, batch_last: bool = False, **kw):
        import torch

        self.bounds = list(bounds)
        n = len(self.bounds) + 1
        shares = shares or ([0.25 / (n - 1)] * (n - 1) + [0.75] if n > 1 else [1.0])
        low, high = torch.cuda.Stream.priority_range()
        self.lanes = []
        for k in range(n):
            stream = torch.cuda.Stream(priority=high if k == 0 else low)
            if k == n - 1 and n > 1 and not batch_last:
                self.lanes.append(SequentialLane(stream=stream, clock=clock, readout=readout))
            else:
                self.lanes.append(FixpointServer(budget_bytes=budget_bytes * shares[k], stream=stream, clock=clock,
                                                 readout=readout, rounds_per_step=rounds_per_step, **kw))

    def lane_for(self, request: ServeRequest) -> int:
        e = len(request.src)
        for k, b in enumerate(self.bounds):
            if e <= b:
                return k
        return len(self.bounds)

    @property
    def completions(self) -> list[Completion]:
        return [c for lane in self.lanes for c in lane.completions]

    @property
    def rounds(self) -> int:
        return sum(lane.rounds for lane in self.lanes)

    def close(self) -> None:
        for lane in self.lanes:
            lane.close()


def serve_laned(requests: list[ServeRequest], server: LanedServer, realtime: bool = True) -> ServeReport:
    """Replays an arrival stream against a LanedServer: the caller's thread
    hands each request to its lane at its arrival time; every lane's thread
    admits, steps and completes its own requests."""
    pending = sorted(requests, key=lambda r: r.arrival_s)
    start = time.perf_counter()
    clock = lambda: time.perf_counter() - start
    for lane in server.lanes:
        lane.clock = clock
    queues = [[] for _ in server.lanes]
    cond = threading.Condition()
    finished = [False]
    errors = []

    def run_lane(k: int, device: int) -> None:
        import torch

        lane = server.lanes[k]
        try:
            torch.cuda.set_device(device)
            while True:
                with cond:
                    while not queues[k] and not lane.active and not finished[0]:
                        cond.wait(0.05)
                    if not queues[k] and not lane.active and finished[0]:
                        return
                    arrived = list(queues[k])
                    queues[k].clear()
                batch = []
                while arrived and lane.can_admit(arrived[0], batch):
                    batch.append(arrived.pop(0))
                if arrived:
                    with cond:
                        queues[k][:0] = arrived
                lane.admit(batch)
                if lane.active:
                    lane.step()
        except BaseException as e:  # surfaced by the caller
            errors.append(e)

    import torch

    device = torch.cuda.current_device()
    threads = [threading.Thread(target=run_lane, args=(k, device), daemon=True) for k in range(len(server.lanes))]
    for t in threads:
        t.start()
    for r in pending:
        if realtime:
            wait = r.arrival_s - clock()
            if wait > 0:
                time.sleep(wait)
        with cond:
            queues[server.lane_for(r)].append(r)
            cond.notify_all()
    with cond:
        finished[0] = True
        cond.notify_all()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return ServeReport(server.completions, clock(), server.rounds)


def _run_alone(req: ServeRequest, stream, readout: str):
    """One request alone through the engine: (path columns, iterations, new rows)."""
    s = np.asarray(req.src, dtype=np.uint32)
    d = np.asarray(req.dst, dtype=np.uint32)
    empty = (np.zeros(0, dtype=np.uint32), np.zeros(0, dtype=np.uint32))
    store = RelationStore(stream)
    store.insert_static(EDB, empty)
    store.insert_recursive(PATH, empty, empty)
    # Same device-side sort/deduplication of the raw edges as the server.
    store.append(EDB, (s, d))
    store.append(PATH, (s, d))
    ex = RecursiveExecutor.compile(transitive_closure_scc(RelationId(PATH), RelationId(EDB)), store)
    summary = ex.run(store)
    if readout == "device":
        import torch

        n = store.rows(PATH)
        with torch.cuda.stream(store.stream):
            path = (torch.empty(max(n, 1), dtype=torch.int32, device="cuda"),
                    torch.empty(max(n, 1), dtype=torch.int32, device="cuda"))
        store.read_into(PATH, 0, path[0], path[1])
        path = (path[0][:n], path[1][:n])
    else:
        path = store.full(PATH)
    ex.close()
    store.close()
    return path, summary.iterations, summary.total_new_rows


def serve_one_at_a_time(requests: list[ServeRequest], stream=None, realtime: bool = True,
                        clock=time.perf_counter, readout: str = "host") -> ServeReport:
    """The baseline: a FIFO loop that runs each request alone through the same engine."""
    pending = sorted(requests, key=lambda r: r.arrival_s)
    start = clock()
    now = lambda: clock() - start
    report = ServeReport()
    for req in pending:
        if realtime and req.arrival_s > now():
            time.sleep(req.arrival_s - now())
        admitted = now()
        path, iterations, new_rows = _run_alone(req, stream, readout)
        report.rounds += iterations
        report.completions.append(Completion(req.request_id, path, iterations, new_rows, req.arrival_s, admitted,
                                             now()))
    report.wall_s = now()
    return report
