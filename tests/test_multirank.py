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


class _OracleBatch:
    """Host stand-in for a rank's BatchEngine: the FP64 oracle per network."""

    def __init__(self, nets, params, math_mode):
        from oracle64 import OracleEngine

        self.o = [OracleEngine(*n.engine_args(), params=p) for n, p in zip(nets, params)]

    def autotune(self, dt):
        pass

    def step_n(self, dt, n):
        return np.stack([o.run(dt, n) for o in self.o], axis=1)  # [steps, nets]

    def close(self):
        pass


SWEEP = dict(num=9, seed=5, n_lo=60, n_hi=300, ks=(4, 6, 8))


def _sweep_worker(rank, world, port, q):
    import torch.distributed as dist

    from leviathan_v1_b200.sharding import run_sweep

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = batch_specs(**SWEEP)
        out = run_sweep(specs, steps=40, tail=10, rank=rank, world_size=world,
                        engine_factory=_OracleBatch)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_gloo_sweep_end_to_end_lands_every_network_in_its_row():
    """run_sweep sharded over two gloo ranks (a host stand-in engine on each)
    gives every rank the whole r(K) table, each network's row equal to that
    network run alone."""
    from leviathan_v1_b200.graphs import build_batch
    from leviathan_v1_b200.sharding import run_sweep

    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sweep_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=150) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    specs = batch_specs(**SWEEP)
    single = run_sweep(specs, steps=40, tail=10, engine_factory=_OracleBatch)
    nets, params = build_batch(specs)
    alone = np.stack([summarize_r(_OracleBatch([n], [p], None).step_n(0.05, 40), 10)[0]
                      for n, p in zip(nets, params)])
    for r in range(world):
        np.testing.assert_array_equal(res[r], single)
    # (mean/std over a [steps, nets] block or one column: summation order only)
    np.testing.assert_allclose(single, alone, rtol=1e-12, atol=1e-15)
    assert len(set(map(tuple, shard_by_edges([s["E"] for s in specs], world)))) == world
