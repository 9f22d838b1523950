"""Autotuner for the executor's launch shapes and thresholds.

The reference fixes its GPU/CPU placement thresholds at compile time for one
device (crates/sparkalog-execution/src/placement.rs:34-38). Here every
launch shape and threshold of the fixpoint (``sparkalog_tuning`` in
``include/sparkalog_b200.h``) is chosen per device by measurement:

* the calibration workload is one transitive-closure fixpoint over a seeded
  Erdos-Renyi graph of the benchmark's family (mean out-degree 0.875, by
  default 4,194,304 nodes: a quarter of the 16.7M-node benchmark graph, so
  one trial takes milliseconds and its rounds have the same shape; the
  shipped choice was calibrated on the full 16,777,216-node graph);
* the search is coordinate descent: each value in turn is swept over its
  candidates with the others held at the best found so far, for a fixed
  number of passes; a trial's cost is the median device time of a few runs
  (fresh store + compile + run + FULL merged into one sorted run, CUDA
  events on the run's stream);
* the choice is saved per device (name and SM count) as JSON. The executor
  applies a saved choice when it is compiled: first the file named by
  ``$SPARKALOG_TUNING``, then the user's cache
  (``~/.cache/sparkalog_b200/``), then the copy shipped in
  ``sparkalog_b200/tuning/``.

Every tuning value gives bit-identical results (the GPU tests run the
fixpoint under several), so tuning changes speed only.

    python -m sparkalog_b200.autotune [--nodes N] [--passes P] [--save PATH | --ship]
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
from pathlib import Path
from typing import Callable

PACKAGE_DIR = Path(__file__).resolve().parent
SHIPPED_DIR = PACKAGE_DIR / "tuning"
CACHE_DIR = Path(os.environ.get("XDG_CACHE_HOME", str(Path.home() / ".cache"))) / "sparkalog_b200"

# Candidate values of each tuning field, in the order the search visits them.
SPACE: dict[str, list[int]] = {
    "dir_rows_log2": [2, 3, 4, 5, 6],
    "group_lanes": [4, 8, 16],
    "group_candidates": [1 << 15, 1 << 17, 1 << 19, 1 << 21],
    "sparse_candidates": [1 << 22, 1 << 24, 1 << 26, 1 << 28],
    "fused_rows_cap": [384, 512, 672, 768],
    "level_ratio": [3, 4, 6, 8],
    "levels": [3, 4],
    "merge_items": [7, 11, 15],
    "bloom_bits": [0, 8, 12, 16],
    "merge_anti_ratio": [0, 2, 4, 8, 16],
    "sparse_items": [2, 3, 4],
    "compact_index": [1, 0],
}


def valid(t: dict) -> bool:
    """The constraint between fields that the library checks too."""
    return t["group_candidates"] <= t["sparse_candidates"]


def coordinate_descent(measure: Callable[[dict], float], start: dict, space: dict[str, list[int]] = SPACE,
                       passes: int = 2) -> tuple[dict, float, list[tuple[dict, float]]]:
    """Minimises measure(tuning) one field at a time.

    Returns (best tuning, its cost, every trial as (tuning, cost)). A trial
    already measured is not repeated; candidates that violate ``valid`` are
    skipped. Ties keep the current value, so the result is deterministic for
    a deterministic ``measure``."""
    best = dict(start)
    seen: dict[tuple, float] = {}
    trials: list[tuple[dict, float]] = []

    def cost(t: dict) -> float:
        key = tuple(sorted(t.items()))
        if key not in seen:
            seen[key] = float(measure(dict(t)))
            trials.append((dict(t), seen[key]))
        return seen[key]

    best_cost = cost(best)
    for _ in range(passes):
        changed = False
        for name, values in space.items():
            for v in values:
                if v == best[name]:
                    continue
                trial = dict(best, **{name: v})
                if not valid(trial):
                    continue
                c = cost(trial)
                if c < best_cost:
                    best, best_cost, changed = trial, c, True
        if not changed:
            break
    return best, best_cost, trials


def device_key() -> str:
    """File-name key of the current CUDA device: its name and SM count."""
    import torch

    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    name = re.sub(r"[^A-Za-z0-9]+", "_", props.name).strip("_")
    return f"{name}_sm{props.multi_processor_count}"


_saved: dict[str, dict | None] = {}


def _read(path: Path) -> dict | None:
    try:
        data = json.loads(path.read_text())
    except (OSError, ValueError):
        return None
    t = data.get("tuning") if isinstance(data, dict) else None
    return dict(t) if isinstance(t, dict) else None


def saved_tuning() -> dict | None:
    """The saved tuning for the current device, or None (then the built-in defaults apply)."""
    env = os.environ.get("SPARKALOG_TUNING")
    if env:
        return _read(Path(env))
    key = device_key()
    if key not in _saved:
        found = None
        for path in (CACHE_DIR / f"{key}.json", SHIPPED_DIR / f"{key}.json"):
            found = _read(path)
            if found is not None:
                break
        _saved[key] = found
    return _saved[key]


def save(tuning: dict, path: Path, meta: dict | None = None) -> Path:
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps({"tuning": tuning, **(meta or {})}, indent=1) + "\n")
    _saved.clear()
    return path


def calibration_measure(nodes: int = 1 << 22, degree: float = 0.875, seed: int = 11, repeats: int = 3):
    """A measure() over one fixpoint of the calibration graph, inputs resident on the device."""
    import numpy as np
    import torch

    from . import generators
    from .recursion import RecursiveExecutor, RelationStore, reserve_device_memory, transitive_closure_scc
    from .relational import RelationId

    src, dst = generators.er_edges(nodes, int(round(nodes * degree)), seed)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()
    e0, e1 = dev(src), dev(dst)
    stream = torch.cuda.current_stream()
    # The pool the fixpoint needs (about 1.5 KB per node), so no trial pays
    # for growing it.
    reserve_device_memory(max(4 << 30, nodes * 1536), stream)
    plan = transitive_closure_scc(RelationId(1), RelationId(0))

    def once(tuning: dict) -> float:
        store = RelationStore(stream)
        try:
            store.insert_static(0, (e0, e1))
            store.insert_recursive(1, (e0, e1), (e0, e1))
            ex = RecursiveExecutor.compile(plan, store)
            ex.set_tuning(tuning)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ex.run(store)
            store.compact(1)
            b.record(stream)
            b.synchronize()
            ex.close()
            return a.elapsed_time(b)
        finally:
            store.close()

    def measure(tuning: dict) -> float:
        once(tuning)  # warm-up (allocations, directory builds)
        return statistics.median(once(tuning) for _ in range(repeats))

    return measure


def defaults() -> dict:
    import ctypes

    from . import _native

    t = _native.TuningC()
    if _native.load().sparkalog_tuning_defaults(ctypes.byref(t)) != 0:
        raise RuntimeError("sparkalog_tuning_defaults failed")
    return t.as_dict()


def tune(nodes: int = 1 << 22, passes: int = 2, repeats: int = 3) -> tuple[dict, float, list]:
    measure = calibration_measure(nodes=nodes, repeats=repeats)
    return coordinate_descent(measure, defaults(), SPACE, passes)


def main() -> None:
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--nodes", type=int, default=1 << 22)
    p.add_argument("--passes", type=int, default=2)
    p.add_argument("--repeats", type=int, default=3)
    g = p.add_mutually_exclusive_group()
    g.add_argument("--save", type=Path, help="write the choice to this file")
    g.add_argument("--ship", action="store_true", help="write it to the package's shipped tuning directory")
    args = p.parse_args()
    start = defaults()
    best, cost, trials = tune(args.nodes, args.passes, args.repeats)
    base = next(c for t, c in trials if t == start)
    meta = {"device": device_key(), "calibration": {"nodes": args.nodes, "degree": 0.875, "seed": 11},
            "ms": cost, "defaults_ms": base, "trials": [{"tuning": t, "ms": c} for t, c in trials]}
    print(json.dumps({"tuning": best, "ms": cost, "defaults_ms": base, "trials": len(trials)}))
    if args.save or args.ship:
        path = args.save or (SHIPPED_DIR / f"{device_key()}.json")
        save(best, path, meta)
        print(f"saved {path}")


if __name__ == "__main__":
    main()
