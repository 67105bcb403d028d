"""One network split over several ranks (the halo engine, halo.py).

CPU: the partition plan's invariants; the data plane (all-gather of tile
partials, halo send/recv, r and the controller from the gathered partials)
as gloo ranks in separate processes and as threads in one process, with the
FP32 NumPy core of ``halo_cpu_core`` standing in for each rank's GPU -- a
partitioned run must equal the unpartitioned run of the same core bit for
bit over 50 steps, including a ``set_theta`` in the middle.  The core
itself is checked against the FP64 oracle.

GPU: the CUDA partition engines (``lev_part_*``) of 2 and 3 partitions on
one device, driven by threads, against the single-GPU engine: bitwise equal
r, phases, weights and gain over 50 steps.  Partitions on one device do not
wait on each other inside kernels (the host orders every exchange), so this
runs safely on one GPU.
"""

import os
import socket
import threading

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import has_gpu
from leviathan_v1_b200.graphs import make_network
from leviathan_v1_b200.halo import (TILE, PartitionedEngine, PartitionPlan,
                                    ThreadExchange)

DT = 0.05
STEPS = 50
KICK_AT = 25


def _net(N=3000, k=12, md=20, seed=4):
    return make_network(N, k, 0.1, md, seed=seed)


# ---------------------------------------------------------------------------
# plan
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_partition_plan_keeps_every_edge(world):
    net = _net()
    plan = PartitionPlan(net.row_ptr, net.col_idx, world)
    rows = []
    for pr in plan.ranks:
        assert pr.row0 % TILE == 0 and pr.tile_off * TILE == pr.row0
        if pr.rank < world - 1:
            assert pr.N % TILE == 0
        rows.append(np.arange(pr.row0, pr.row1))
        # local CSR is the own rows' slice; columns map back to global ids
        assert pr.row_ptr[0] == 0 and pr.row_ptr[-1] == pr.edge1 - pr.edge0
        loc = pr.col_idx.astype(np.int64)
        halo_ext = np.concatenate([pr.halo, [-1]])  # -1 never matches
        glob = np.where(loc < pr.N, loc + pr.row0, halo_ext[np.clip(loc - pr.N, 0, pr.n_halo)])
        np.testing.assert_array_equal(glob, net.col_idx[pr.edge0:pr.edge1])
        assert np.all((pr.halo < pr.row0) | (pr.halo >= pr.row1))
        assert np.all(np.diff(pr.halo) > 0)
        for p, pos in pr.recv.items():
            b0, b1 = plan.bounds[p]
            assert np.all((pr.halo[pos] >= b0) & (pr.halo[pos] < b1))
            assert np.all(np.diff(pos) == 1)  # a contiguous block of the halo
            send = plan.rank(p).send[pr.rank]
            np.testing.assert_array_equal(send + b0, pr.halo[pos])
        assert sum(v.size for v in pr.recv.values()) == pr.n_halo
    np.testing.assert_array_equal(np.concatenate(rows), np.arange(net.N))
    assert sum(pr.edge1 - pr.edge0 for pr in plan.ranks) == net.E


def test_partition_plan_rejects_empty_partitions():
    net = _net(N=700)  # 3 tiles
    PartitionPlan(net.row_ptr, net.col_idx, 3)
    with pytest.raises(ValueError):
        PartitionPlan(net.row_ptr, net.col_idx, 4)


# ---------------------------------------------------------------------------
# CPU data plane
# ---------------------------------------------------------------------------
def _run(engine, net):
    """50 steps with a set_theta (phase kick) after step KICK_AT."""
    r1 = engine.step_n(DT, KICK_AT)
    th = engine.gather_theta()
    th[::7] = np.remainder(th[::7] + np.float32(1.5), np.float32(2 * np.pi))
    engine.set_theta(th)
    r2 = engine.step_n(DT, STEPS - KICK_AT)
    return dict(r=np.concatenate([r1, r2]), theta=engine.gather_theta(),
                w=engine.get_weights(), g=engine.get_gain())


def _unpartitioned(net, core):
    from leviathan_v1_b200.halo import _ThreadRank  # noqa: F401

    ex = ThreadExchange(1).bind(0)
    e = PartitionedEngine(0, 1, *net.engine_args(), exchange=ex, core=core)
    out = _run(e, net)
    e.close()
    return out


def test_cpu_core_matches_fp64_oracle():
    from halo_cpu_core import CpuPartitionCore
    from oracle64 import OracleEngine, circular_distance

    net = _net()
    ex = ThreadExchange(1).bind(0)
    e = PartitionedEngine(0, 1, *net.engine_args(), exchange=ex, core=CpuPartitionCore)
    r = e.step_n(DT, 30)
    o = OracleEngine(*net.engine_args())
    ro = o.run(DT, 30)
    assert np.abs(r - ro).max() < 1e-4
    assert circular_distance(e.gather_theta(), o.theta).max() < 1e-3
    assert np.abs(e.get_weights() - o.w).max() < 1e-4


def _threads(net, world, core, pairs=None):
    hub = ThreadExchange(world)
    plan = PartitionPlan(net.row_ptr, net.col_idx, world)
    res, errs = {}, []

    def work(r):
        try:
            e = PartitionedEngine(r, world, *net.engine_args(), exchange=hub.bind(r),
                                  core=core, plan=plan)
            res[f"pairs{r}"] = e._pairs
            if pairs is not None:
                e.set_pair_mode(pairs)
            res[r] = _run(e, net)
            e.close()
        except BaseException as exc:  # report, and release the others
            errs.append(exc)
            hub._bar.abort()

    ts = [threading.Thread(target=work, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    if errs:
        raise errs[0]
    return res


def _check_equal(res, ref, world):
    w = np.concatenate([res[r]["w"] for r in range(world)])
    for r in range(world):
        np.testing.assert_array_equal(res[r]["r"], ref["r"])
        np.testing.assert_array_equal(res[r]["theta"], ref["theta"])
        assert res[r]["g"] == ref["g"]
    np.testing.assert_array_equal(w, ref["w"])


@pytest.mark.parametrize("pairs", [True, False], ids=["pairs", "single"])
def test_threads_partitioned_equals_unpartitioned_cpu(pairs):
    from halo_cpu_core import CpuPartitionCore

    net = _net()
    ref = _unpartitioned(net, CpuPartitionCore)
    res = _threads(net, 4, CpuPartitionCore, pairs)
    assert all(res[f"pairs{r}"] for r in range(4))  # no zero delay anywhere
    _check_equal(res, ref, 4)


def test_ranks_agree_on_pairs():
    """One zero delay in rank 0's rows only: every rank steps one step per
    launch (they issue the same collectives), and the run is unchanged."""
    from halo_cpu_core import CpuPartitionCore

    net = _net()
    net.delays = net.delays.copy()
    net.delays[5] = 0
    ref = _unpartitioned(net, CpuPartitionCore)
    res = _threads(net, 3, CpuPartitionCore)
    assert not any(res[f"pairs{r}"] for r in range(3))
    _check_equal(res, ref, 3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, q):
    import torch.distributed as dist

    from halo_cpu_core import CpuPartitionCore
    from leviathan_v1_b200.halo import DistExchange

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        net = _net()
        e = PartitionedEngine(rank, world, *net.engine_args(), exchange=DistExchange(),
                              core=CpuPartitionCore)
        q.put((rank, _run(e, net)))
        e.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
@pytest.mark.parametrize("world", [2, 3])
def test_gloo_partitioned_equals_unpartitioned(world):
    from halo_cpu_core import CpuPartitionCore

    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=200) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    _check_equal(res, _unpartitioned(_net(), CpuPartitionCore), world)


# ---------------------------------------------------------------------------
# GPU: CUDA partition engines on one device
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("pairs", [True, False], ids=["pairs", "single"])
@pytest.mark.parametrize("world,math_mode", [(2, "reference"), (3, "accurate")])
def test_cuda_partitions_equal_single_engine(world, math_mode, pairs):
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200 import LeviathanEngine
    from leviathan_v1_b200.halo import CudaPartition

    net = make_network(20_000, 16, 0.1, 30, seed=11)
    eng = LeviathanEngine(*net.engine_args(), math_mode=math_mode)
    r1 = np.array([eng.step(DT) for _ in range(KICK_AT)], np.float32)
    th = eng.get_theta()
    th[::7] = np.remainder(th[::7] + np.float32(1.5), np.float32(2 * np.pi))
    eng.set_theta(th)
    r2 = np.array([eng.step(DT) for _ in range(STEPS - KICK_AT)], np.float32)
    ref = dict(r=np.concatenate([r1, r2]), theta=eng.get_theta(), w=eng.get_weights(),
               g=eng.get_gain())
    eng.close()

    hub = ThreadExchange(world)
    plan = PartitionPlan(net.row_ptr, net.col_idx, world)
    assert all(pr.n_halo > 0 for pr in plan.ranks)
    res, errs = {}, []

    def work(r):
        try:
            import torch

            torch.cuda.set_device(0)
            e = PartitionedEngine(r, world, *net.engine_args(), exchange=hub.bind(r),
                                  plan=plan, core=CudaPartition, math_mode=math_mode)
            assert e._pairs  # no zero delay: two steps per pair of launches
            e.set_pair_mode(pairs)
            res[r] = _run(e, net)
            e.close()
        except BaseException as exc:
            errs.append(exc)
            hub._bar.abort()

    ts = [threading.Thread(target=work, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    if errs:
        raise errs[0]
    _check_equal(res, ref, world)
