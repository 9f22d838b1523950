"""Multi-rank x-range sharding on CPU (gloo, world size 2).

Each rank closes its x range of the seed against the replicated EDB (the CPU
oracle stands in for the per-GPU engine), then the ranks combine iteration
counts and new rows with all-reduces and gather their FULL parts. The union
must equal the single-rank fixpoint, and the combined counts its counts.
"""

import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from sparkalog_b200 import generators, sharding


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nodes, edges, seed, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        src, dst = generators.er_edges(nodes, edges, seed)
        s0, s1 = sharding.partition_seed(src, dst, nodes, rank, world)
        st = oracle.Store()
        st.insert_static(0, (src, dst))
        st.insert_recursive(1, (s0, s1), (s0, s1))
        it, new = st.run_scc([1], [oracle.tc_rule(1, 0)])
        g_it, g_new = sharding.combine_summaries(it, new)
        part = st.full(1)
        gathered = [None] * world
        dist.all_gather_object(gathered, (part[0].tolist(), part[1].tolist()))
        if rank == 0:
            out.put((g_it, g_new, gathered))
    finally:
        dist.destroy_process_group()


def test_two_rank_partition_matches_single_rank():
    nodes, edges, seed = 3000, 2800, 13
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, nodes, edges, seed, q)) for r in range(2)]
    for p in procs:
        p.start()
    g_it, g_new, parts = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    src, dst = generators.er_edges(nodes, edges, seed)
    (w0, w1), it, new = oracle.transitive_closure(src, dst)
    assert g_it == it
    assert g_new == new
    f0 = np.concatenate([np.array(p[0], dtype=np.uint32) for p in parts])
    f1 = np.concatenate([np.array(p[1], dtype=np.uint32) for p in parts])
    assert np.array_equal(f0, w0) and np.array_equal(f1, w1)


def test_x_ranges_tile_the_nodes():
    for world in (1, 2, 3, 8):
        ranges = [sharding.x_range(1001, r, world) for r in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == 1001
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))


def test_balanced_bounds_split_no_x():
    src = np.sort(np.random.default_rng(3).integers(0, 50, 10_000)).astype(np.uint32)
    for world in (2, 3, 7):
        b = sharding.balanced_bounds(src, 50, world)
        assert b[0] == 0 and b[-1] == 50 and b == sorted(b)
        rows = [len(sharding.partition_seed(src, src, 50, r, world, balanced=True)[0]) for r in range(world)]
        assert sum(rows) == len(src)
