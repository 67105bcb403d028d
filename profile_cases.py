"""Representative workloads of each kernel, for profilers (measurement
tooling beside bench.py; not part of the package).

    python profile_cases.py step      [--N 1000000 --k 32 --steps 5]
    python profile_cases.py cluster   [--N 1000 --k 20 --steps 200]
    python profile_cases.py grid      [--N 10000 --k 20 --steps 200]
    python profile_cases.py batched   [--batch 128 --steps 20 --pair -1]
    python profile_cases.py adjoint   [--N 200000 --k 32 --T 100]
    python profile_cases.py adjgrid   [--N 10000 --k 20 --T 200]
    python profile_cases.py reservoir [--N 20000 --batch 8 --T 60]
    python profile_cases.py e2e       [--N 1000000 --k 32 --steps 500]

Each runs a short, fixed amount of work on the current CUDA device (graphs
built on the device, seeded) and prints one JSON line of timings; sizes are
chosen so that a full-metric capture of one launch stays within a few GB of
device memory.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def _sync():
    import torch

    torch.cuda.synchronize()


def case_step(a):
    from leviathan_v1_b200.engine import LeviathanEngine
    from leviathan_v1_b200.graphs import make_network_gpu

    net = make_network_gpu(a.N, a.k, 0.1, a.max_delay, a.seed)
    e = LeviathanEngine(*net.engine_args())
    if a.pair >= 0:  # the two-steps-per-launch variant the autotuner picks
        for c in range(3):
            e.set_pair_variant(c, a.pair)
    e.step_n(0.05, 3)
    _sync()
    t = time.perf_counter()
    e.step_n(0.05, a.steps)
    dt = time.perf_counter() - t
    e.close()
    return dict(case="step", N=a.N, E=net.E, steps=a.steps, s=dt, pair=a.pair)


def case_cluster(a):
    from leviathan_v1_b200.engine import LeviathanEngine
    from leviathan_v1_b200.graphs import make_network_gpu

    net = make_network_gpu(a.N, a.k, 0.1, a.max_delay, a.seed)
    e = LeviathanEngine(*net.engine_args())
    e.set_cluster_mode(True)
    info = e.cluster_info()
    e.step_n(0.05, 3)
    _sync()
    t = time.perf_counter()
    e.step_n(0.05, a.steps)
    dt = time.perf_counter() - t
    e.close()
    return dict(case="cluster", N=a.N, E=net.E, steps=a.steps, s=dt, cluster=info)


def case_grid(a):
    from leviathan_v1_b200.engine import LeviathanEngine
    from leviathan_v1_b200.graphs import make_network_gpu

    net = make_network_gpu(a.N, a.k, 0.1, a.max_delay, a.seed)
    e = LeviathanEngine(*net.engine_args())
    e.set_cluster_mode(False)
    e.set_grid_mode(True, 64)
    info = e.grid_info()
    e.step_n(0.05, 3)
    _sync()
    t = time.perf_counter()
    e.step_n(0.05, a.steps)
    dt = time.perf_counter() - t
    e.close()
    return dict(case="grid", N=a.N, E=net.E, steps=a.steps, s=dt, grid=info)


def case_batched(a):
    """The first `batch` networks of the 512-network coupling sweep (N
    log-uniform in [500, 5e4], k in {8, 16, 20, 32}, delays [1,50], K swept,
    controller off), autotuned, then `steps` steps in step blocks.  `pair` >= 0
    sets that two-steps-per-launch variant for every class after the
    autotuner (under a profiler the autotuner's timings do not hold)."""
    from leviathan_v1_b200.engine import BatchEngine
    from leviathan_v1_b200.graphs import batch_specs, build_batch

    specs = batch_specs(512, seed=0)[:a.batch]
    nets, params = build_batch(specs)
    e = BatchEngine([n.as_dict() for n in nets], params=params)
    e.autotune(0.05, trial_steps=3)
    if a.pair >= 0:
        for c in range(3):
            e.set_pair_variant(c, a.pair)
    e.step_n(0.05, 3)
    _sync()
    t = time.perf_counter()
    e.step_n(0.05, a.steps)
    dt = time.perf_counter() - t
    out = dict(case="batched", networks=len(nets), N=sum(n.N for n in nets),
               E=sum(n.E for n in nets), steps=a.steps, s=dt, pair_info=e.pair_info())
    e.close()
    return out


def case_adjoint(a):
    import torch

    from leviathan_v1_b200.adjoint import Adjoint, simulate
    from leviathan_v1_b200.engine import LeviathanEngine
    from leviathan_v1_b200.graphs import make_network_gpu

    net = make_network_gpu(a.N, a.k, 0.1, a.max_delay, a.seed)
    eng = LeviathanEngine(*net.engine_args(), math_mode="accurate")
    adj = Adjoint(eng, segment=a.segment, max_steps=a.T)
    om = torch.tensor(net.omega, device="cuda", requires_grad=True)
    w0 = torch.tensor(net.weights, device="cuda", requires_grad=True)
    K = torch.full((1,), 1.5, device="cuda", requires_grad=True)
    _sync()
    t = time.perf_counter()
    r = simulate(adj, om, w0, K, a.T, 0.05)
    (r ** 2).mean().backward()
    _sync()
    dt = time.perf_counter() - t
    out = dict(case=a.case, N=a.N, E=net.E, T=a.T, segment=a.segment, s=dt,
               device_bytes=adj.device_bytes, grid=adj.grid_info())
    adj.close()
    eng.close()
    return out


def case_reservoir(a):
    import torch

    from leviathan_v1_b200.graphs import make_network_gpu
    from leviathan_v1_b200.reservoir import DifferentiableReservoir, make_inputs

    net = make_network_gpu(a.N, a.k, 0.1, a.max_delay, a.seed)
    m = DifferentiableReservoir(net, a.batch, n_input=min(256, a.N // 4), T=a.T,
                                segment=a.segment)
    x = torch.tensor(make_inputs(a.batch, a.T), device="cuda")
    _sync()
    t = time.perf_counter()
    y, r = m(x)
    m.loss(y, x, 10).backward()
    _sync()
    dt = time.perf_counter() - t
    out = dict(case="reservoir", N=a.N, batch=a.batch, T=a.T, s=dt,
               device_bytes=m.adj.device_bytes)
    m.close()
    return out


def case_e2e(a):
    """Breakdown of the whole job through the public API: engine
    construction from host arrays, K synchronous steps, snapshot."""
    from leviathan_v1_b200.engine import LeviathanEngine
    from leviathan_v1_b200.graphs import make_network_gpu

    net = make_network_gpu(a.N, a.k, 0.1, a.max_delay, a.seed)
    e = LeviathanEngine(*net.engine_args())  # warm-up: context, module load
    e.close()
    _sync()
    t0 = time.perf_counter()
    e = LeviathanEngine(*net.engine_args())
    _sync()
    t1 = time.perf_counter()
    for _ in range(a.steps):
        e.step(0.05)
    t2 = time.perf_counter()
    e.get_theta()
    t3 = time.perf_counter()
    e.step_n(0.05, a.steps)
    t4 = time.perf_counter()
    e.close()
    return dict(case="e2e", N=a.N, E=net.E, steps=a.steps, construct_s=t1 - t0,
                steps_s=t2 - t1, per_step_us=(t2 - t1) / a.steps * 1e6,
                snapshot_s=t3 - t2, step_n_per_step_us=(t4 - t3) / a.steps * 1e6)


CASES = dict(step=case_step, cluster=case_cluster, grid=case_grid, batched=case_batched,
             adjoint=case_adjoint,
             adjgrid=case_adjoint,
             reservoir=case_reservoir, e2e=case_e2e)
DEFAULTS = dict(step=dict(N=1_000_000, k=32, max_delay=64, steps=5, pair=-1),
                cluster=dict(N=1000, k=20, max_delay=50, steps=200),
                grid=dict(N=10_000, k=20, max_delay=50, steps=200),
                batched=dict(N=0, k=0, max_delay=50, batch=128, steps=20, pair=-1),
                adjgrid=dict(N=10_000, k=20, max_delay=50, T=200),
                adjoint=dict(N=200_000, k=32, max_delay=50, T=100),
                reservoir=dict(N=20_000, k=20, max_delay=50, T=60, batch=8),
                e2e=dict(N=1_000_000, k=32, max_delay=64, steps=500))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=sorted(CASES))
    for name, typ in (("N", int), ("k", int), ("max_delay", int), ("steps", int),
                      ("T", int), ("batch", int), ("segment", int), ("seed", int),
                      ("pair", int)):
        ap.add_argument(f"--{name}", type=typ, default=None)
    a = ap.parse_args(argv)
    d = dict(DEFAULTS[a.case], segment=50, seed=0, case=a.case)
    for k_, v in vars(a).items():
        if v is not None:
            d[k_] = v
    for k_, v in d.items():
        setattr(a, k_, v)
    print(json.dumps(CASES[a.case](a)), flush=True)


if __name__ == "__main__":
    main()
