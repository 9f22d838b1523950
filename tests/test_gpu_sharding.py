"""The engine under x-range partitioning, on one GPU.

Each partition (the seed rows whose x lies in one rank's range, against the
whole replicated EDB) runs to its own fixpoint through the device engine, one
after the other on the same GPU. Concatenated in rank order, their FULLs must
equal the single-run FULL, the largest per-partition iteration count the
single run's count, and the new rows must add up (what the multi-GPU bench
combines with its final all-reduce). Equal node ranges and seed-balanced
ranges (for a skewed graph) are both checked.
"""

import numpy as np
import pytest

import oracle
from sparkalog_b200 import generators, sharding

pytestmark = pytest.mark.gpu


def _run(src, dst, s0, s1):
    from sparkalog_b200.recursion import RecursiveExecutor, RelationStore, transitive_closure_scc
    from sparkalog_b200.relational import RelationId

    store = RelationStore()
    store.insert_static(0, (src, dst))
    store.insert_recursive(1, (s0, s1), (s0, s1))
    ex = RecursiveExecutor.compile(transitive_closure_scc(RelationId(1), RelationId(0)), store)
    summary = ex.run(store)
    ex.close()
    full = store.full(1)
    store.close()
    return full, summary.iterations, summary.total_new_rows


def _skewed(nodes, edges, seed):
    """An ER graph plus a hub: every tenth node points at node 0's block."""
    src, dst = generators.er_edges(nodes, edges, seed)
    hub_src = np.arange(0, nodes, 10, dtype=np.uint32)
    hub_dst = (hub_src % 97).astype(np.uint32)
    return oracle.btree_pairs(np.concatenate([src, hub_src]), np.concatenate([dst, hub_dst]))


@pytest.mark.parametrize("world,balanced,skewed", [(2, False, False), (4, False, False), (4, True, True)])
def test_partitions_concatenate_to_the_single_run(cuda, world, balanced, skewed):
    nodes, edges, seed = 400_000, 350_000, 31
    src, dst = _skewed(nodes, edges, seed) if skewed else generators.er_edges(nodes, edges, seed)
    (w0, w1), it, new = _run(src, dst, src, dst)
    parts, its, news, seeds = [], [], [], []
    for rank in range(world):
        s0, s1 = sharding.partition_seed(src, dst, nodes, rank, world, balanced=balanced)
        seeds.append(len(s0))
        (f0, f1), i, n = _run(src, dst, s0, s1)
        parts.append((f0, f1))
        its.append(i)
        news.append(n)
    assert sum(seeds) == len(src)
    assert max(its) == it and sum(news) == new
    assert np.array_equal(np.concatenate([p[0] for p in parts]), w0)
    assert np.array_equal(np.concatenate([p[1] for p in parts]), w1)
    if balanced:
        assert max(seeds) <= 1.2 * len(src) / world
