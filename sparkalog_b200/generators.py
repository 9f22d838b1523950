"""Seeded synthetic workloads for the transitive-closure pipeline.

There is no public benchmark suite for this path, so every workload is a
deterministic function of its seed:

* ``er_edges`` — a directed Erdos-Renyi graph: candidate j is
  (hi32(z(2j)) * n >> 32, hi32(z(2j+1)) * n >> 32) with z the splitmix64
  output for counter i (state = seed + (i + 1) * 0x9E3779B97F4A7C15);
  self-loops are rejected and the first ``n_edges`` distinct candidates in j
  order are kept. Returned sorted by (src, dst), the order execute_binary
  gives an EDB. The oracle restates the same generator in C, and a test
  checks that both agree.
* ``batched_instances`` — independent TC instances with node counts
  log-uniform in [64, 16384] and mean out-degree uniform in [0.5, 1.2].
* ``served_requests`` — a Poisson arrival stream of TC requests with edge
  counts log-uniform in [1e3, 4e6] and mean out-degree uniform in [0.6, 0.95].
* ``uniform_pairs`` — deduplicated uniform pairs (the candidate relation of
  the stratified-negation workload).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)
MASK32 = np.uint64(0xFFFFFFFF)


def splitmix64(seed: int, counters: np.ndarray) -> np.ndarray:
    """splitmix64 outputs for the given counters (vectorised, wrapping u64 arithmetic)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + (counters.astype(np.uint64) + np.uint64(1)) * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def _bounded(z: np.ndarray, n: int) -> np.ndarray:
    return ((z >> np.uint64(32)) * np.uint64(n)) >> np.uint64(32)


def unit_float(seed: int, counters: np.ndarray) -> np.ndarray:
    """Uniform [0, 1) doubles from the top 53 bits of splitmix64."""
    return (splitmix64(seed, counters) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def er_edges_packed(n_nodes: int, n_edges: int, seed: int) -> np.ndarray:
    """Sorted packed (src << 32 | dst) keys of the seeded ER edge set."""
    if n_nodes < 2 or n_edges <= 0:
        return np.zeros(0, dtype=np.uint64)
    n_edges = min(n_edges, n_nodes * (n_nodes - 1))
    parts = []
    j0 = 0
    while True:
        have = sum(len(p) for p in parts)
        block = max(int((n_edges - have) * 1.25) + 4096, 4096) if have < n_edges else max(n_edges // 4, 4096)
        j = np.arange(j0, j0 + block, dtype=np.uint64)
        u = _bounded(splitmix64(seed, 2 * j), n_nodes)
        v = _bounded(splitmix64(seed, 2 * j + np.uint64(1)), n_nodes)
        keep = u != v
        parts.append((u[keep] << np.uint64(32)) | v[keep])
        j0 += block
        cand = np.concatenate(parts) if len(parts) > 1 else parts[0]
        uniq, first = np.unique(cand, return_index=True)
        if len(uniq) >= n_edges:
            order = np.argsort(first, kind="stable")[:n_edges]
            return np.sort(uniq[order])
        parts = [cand]


def er_edges(n_nodes: int, n_edges: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """(src, dst) u32 columns of the seeded ER graph, sorted by (src, dst)."""
    packed = er_edges_packed(n_nodes, n_edges, seed)
    return (packed >> np.uint64(32)).astype(np.uint32), (packed & MASK32).astype(np.uint32)


def uniform_pairs(n_nodes: int, n_pairs: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """``n_pairs`` uniform pairs over [0, n_nodes)^2 (self-pairs allowed), deduplicated and sorted."""
    j = np.arange(n_pairs, dtype=np.uint64)
    u = _bounded(splitmix64(seed, 2 * j), n_nodes)
    v = _bounded(splitmix64(seed, 2 * j + np.uint64(1)), n_nodes)
    packed = np.unique((u << np.uint64(32)) | v)
    return (packed >> np.uint64(32)).astype(np.uint32), (packed & MASK32).astype(np.uint32)


@dataclass
class Instance:
    nodes: int
    degree: float
    edges: int
    seed: int


def batched_instances(count: int, base_seed: int, n_min: int = 64, n_max: int = 16384,
                      d_min: float = 0.5, d_max: float = 1.2) -> list[Instance]:
    """Parameters of ``count`` independent ER instances (node counts log-uniform, degrees uniform)."""
    i = np.arange(count, dtype=np.uint64)
    u_n = unit_float(base_seed, 3 * i)
    u_d = unit_float(base_seed, 3 * i + np.uint64(1))
    seeds = splitmix64(base_seed, 3 * i + np.uint64(2))
    ratio = np.log(n_max / n_min)
    nodes = np.clip(np.rint(n_min * np.exp(u_n * ratio)), n_min, n_max).astype(np.int64)
    degree = d_min + (d_max - d_min) * u_d
    edges = np.minimum(np.rint(nodes * degree).astype(np.int64), nodes * (nodes - 1))
    return [Instance(int(n), float(d), int(e), int(s)) for n, d, e, s in zip(nodes, degree, edges, seeds)]


@dataclass
class Request:
    arrival_s: float
    nodes: int
    degree: float
    edges: int
    seed: int


def served_requests(count: int, rate_per_s: float, base_seed: int, e_min: float = 1e3, e_max: float = 4e6,
                    d_min: float = 0.6, d_max: float = 0.95) -> list[Request]:
    """A seeded Poisson stream of TC requests."""
    i = np.arange(count, dtype=np.uint64)
    gaps = -np.log1p(-unit_float(base_seed, 4 * i)) / rate_per_s
    arrivals = np.cumsum(gaps)
    u_e = unit_float(base_seed, 4 * i + np.uint64(1))
    u_d = unit_float(base_seed, 4 * i + np.uint64(2))
    seeds = splitmix64(base_seed, 4 * i + np.uint64(3))
    edges = np.rint(e_min * np.exp(u_e * np.log(e_max / e_min))).astype(np.int64)
    degree = d_min + (d_max - d_min) * u_d
    nodes = np.maximum(np.rint(edges / degree).astype(np.int64), 2)
    return [Request(float(a), int(n), float(d), int(e), int(s))
            for a, n, d, e, s in zip(arrivals, nodes, degree, edges, seeds)]


# The five workloads of the benchmark, by name.
CONFIGS = {
    "er_2000_8000": dict(nodes=2_000, edges=8_000, seed=1),
    "er_16m_14_68m": dict(nodes=16_777_216, edges=14_680_064, seed=2),
    "negation_8m": dict(nodes=8_388_608, edges=7_340_032, seed=5, cand_pairs=50_000_000, cand_seed=55),
}
