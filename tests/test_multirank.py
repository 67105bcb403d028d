"""Multi-rank host logic on CPU (gloo, world_size 2): sharding of batched
sweeps, result gathering, and the bench's max/sum over ranks."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from leviathan_v1_b200.graphs import batch_specs
from leviathan_v1_b200.sharding import gather_results, shard_by_edges, summarize_r


def test_shard_by_edges_covers_all_once_and_balances():
    specs = batch_specs(512, seed=0)
    E = [s["E"] for s in specs]
    for ws in (1, 2, 3, 8):
        shards = shard_by_edges(E, ws)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(512))
        loads = [sum(E[i] for i in s) for s in shards]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(E) / ws + max(E)
        assert shard_by_edges(E, ws) == shards  # deterministic


def test_shard_more_ranks_than_networks():
    shards = shard_by_edges([5, 3], 4)
    assert sorted(len(s) for s in shards) == [0, 0, 1, 1]


def test_summarize_r():
    r = np.arange(20, dtype=np.float64).reshape(10, 2)
    s = summarize_r(r, 4)
    assert np.allclose(s[:, 0], r[-4:].mean(axis=0))
    assert np.allclose(s[:, 1], r[-4:].std(axis=0))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = batch_specs(37, seed=3)
        shards = shard_by_edges([s["E"] for s in specs], world)
        mine = shards[rank]
        local = np.array([[float(i), float(rank)] for i in mine]).reshape(-1, 2)
        out = gather_results(mine, local, len(specs))
        # the bench's max / sum over ranks
        import sys
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        import bench

        mx = bench.max_over_ranks(10.0 + rank, world)
        sm = bench.sum_over_ranks(1.0 + rank, world)
        q.put((rank, out, mx, sm))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_gloo_two_ranks_gather_and_reduce():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    specs = batch_specs(37, seed=3)
    shards = shard_by_edges([s["E"] for s in specs], world)
    for rank, out, mx, sm in res:
        assert out.shape == (37, 2)
        assert np.array_equal(out[:, 0], np.arange(37))
        for r, s in enumerate(shards):
            assert np.all(out[s, 1] == r)
        assert mx == 11.0 and sm == 3.0
