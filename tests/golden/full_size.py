"""Oracle digests of the full-size workloads (configs 2, 3 and 5).

The oracle needs minutes per full-size fixpoint (config 2: 86 rounds,
117,351,424 rows of FULL, about four minutes on eight cores) and its outputs
are gigabytes, so the GPU parity tests compare the device's outputs with
digests of the oracle's outputs made by this script and committed beside it
as ``full_size_digests.json``:

* a relation's digest is the SHA-256 of its two sorted ``u32`` columns
  (first column's bytes, then second column's, little-endian), so equal
  digests mean equal rows in equal order;
* the iteration counts and derived-row counts of every recursive SCC are
  stored as numbers.

Workloads (the same seeded generators the bench uses):

* ``er_16m``: TC of the 16,777,216-node / 14,680,064-edge ER graph, seed 2;
* ``negation_8m``: TC of the 8,388,608-node / 7,340,032-edge ER graph, seed 5,
  then ``unreached = distinct(cand) - path`` for 5.0e7 raw uniform candidate
  pairs (splitmix64 seed 55, duplicates kept in the raw stream);
* ``batched_4096``: 4,096 independent instances from
  ``generators.batched_instances(4096, 3)``; one digest, iteration count and
  derived-row count per instance.

Regenerate with ``python tests/golden/full_size.py`` (needs only the CPU).
"""

from __future__ import annotations

import hashlib
import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
DIGESTS = HERE / "full_size_digests.json"

ER_16M = dict(nodes=16_777_216, edges=14_680_064, seed=2)
NEGATION_8M = dict(nodes=8_388_608, edges=7_340_032, seed=5, cand_pairs=50_000_000, cand_seed=55)
BATCHED = dict(count=4096, base_seed=3)


def pair_digest(first, second) -> str:
    """SHA-256 of the two u32 columns (first's bytes, then second's)."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(first, dtype=np.uint32).tobytes())
    h.update(np.ascontiguousarray(second, dtype=np.uint32).tobytes())
    return h.hexdigest()


def negation_candidates(nodes: int, count: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """The raw candidate stream of the negation workload (duplicates kept)."""
    sys.path.insert(0, str(ROOT))
    from sparkalog_b200 import generators

    j = np.arange(count, dtype=np.uint64)
    c0 = generators._bounded(generators.splitmix64(seed, 2 * j), nodes).astype(np.uint32)
    c1 = generators._bounded(generators.splitmix64(seed, 2 * j + np.uint64(1)), nodes).astype(np.uint32)
    return c0, c1


def batched_edges():
    sys.path.insert(0, str(ROOT))
    from sparkalog_b200 import generators

    params = generators.batched_instances(BATCHED["count"], BATCHED["base_seed"])
    return [generators.er_edges(p.nodes, p.edges, p.seed) for p in params]


def _instance_digest(args):
    sys.path.insert(0, str(ROOT))
    import oracle

    k, src, dst = args
    (f0, f1), it, new = oracle.transitive_closure(src, dst, threads=1)
    return k, int(it), int(new), int(len(f0)), pair_digest(f0, f1)


def main() -> None:
    sys.path.insert(0, str(ROOT))
    import oracle
    from sparkalog_b200 import generators

    threads = os.cpu_count() or 1
    out = {"what": "oracle digests of the full-size workloads; see tests/golden/full_size.py"}
    t = time.time()
    src, dst = generators.er_edges(ER_16M["nodes"], ER_16M["edges"], ER_16M["seed"])
    (f0, f1), it, new = oracle.transitive_closure(src, dst, threads=threads)
    out["er_16m"] = dict(ER_16M, iterations=int(it), new_rows=int(new), rows=int(len(f0)),
                         digest=pair_digest(f0, f1))
    print("er_16m", time.time() - t, out["er_16m"], flush=True)
    del f0, f1, src, dst

    t = time.time()
    p = NEGATION_8M
    src, dst = generators.er_edges(p["nodes"], p["edges"], p["seed"])
    (f0, f1), it, new = oracle.transitive_closure(src, dst, threads=threads)
    c0, c1 = negation_candidates(p["nodes"], p["cand_pairs"], p["cand_seed"])
    u0, u1 = oracle.anti_join(oracle.distinct((c0, c1), threads=threads), (f0, f1), threads=threads)
    out["negation_8m"] = dict(p, iterations=int(it), new_rows=int(new), path_rows=int(len(f0)),
                              path_digest=pair_digest(f0, f1), unreached_rows=int(len(u0)),
                              unreached_digest=pair_digest(u0, u1))
    print("negation_8m", time.time() - t, out["negation_8m"], flush=True)
    del f0, f1, u0, u1, c0, c1

    t = time.time()
    inst = batched_edges()
    jobs = [(k, s, d) for k, (s, d) in enumerate(inst)]
    # Largest instances first so the pool's tail is short.
    jobs.sort(key=lambda j: -len(j[1]))
    rows = [None] * len(inst)
    with mp.get_context("spawn").Pool(threads) as pool:
        for k, it, new, n, digest in pool.imap_unordered(_instance_digest, jobs, chunksize=4):
            rows[k] = [it, new, n, digest]
    out["batched_4096"] = dict(BATCHED, columns=["iterations", "new_rows", "rows", "digest"], instances=rows,
                               new_rows=int(sum(r[1] for r in rows)))
    print("batched_4096", time.time() - t, out["batched_4096"]["new_rows"], flush=True)
    DIGESTS.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
