#!/usr/bin/env python3
"""Benchmark of the LEVIATHAN core engine step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one engine step of the whole network): plain engine
at scale -- seeded Watts-Strogatz N = 1,000,000, k = 32, p = 0.1 (E = 32 M
directed edges), delays uniform in [1, 64], omega ~ N(0,1), theta ~ U[0,2pi),
w ~ U[0,1), dt = 0.05, reference parameter defaults, controller on.
Inputs (1.2 GB resident) exceed the 126 MB L2, so no flush is needed.

Metric: edge-updates/s = E x steps / elapsed.
* ``value``   -- device-resident throughput: K steps replayed from CUDA
  graphs, timed with CUDA events on the engine stream, max over ranks.
* ``e2e``     -- the whole job through the public API with host buffers:
  ``LeviathanEngine(...)`` from host arrays (H2D), ``step_n(dt, K)``
  returning r of every step to the host (the block form
  ``LeviathanObservatory.run_baseline`` uses), ``get_theta()`` (D2H), wall
  clock; ``e2e.per_step_calls`` is the same job with K x ``step(dt)``.
* ``roofline`` -- the dominant kernel (two steps per launch: pair_kernel) at
  its algorithmic bytes per launch over its mean launch duration (CUDA
  events on the engine stream), against the measured HBM copy peak; the
  per-step figure of the whole launch sequence is in ``step_sequence``.
* ``--impl reference`` runs the reference engine itself (its
  leviathan_kernel.cu built from the reference sources for sm_100a, and its
  stock 86;90 build, in oracle/_ref) through its C ABI on the same GPU (the
  reference has no CPU implementation of the path): ``value`` is K steps
  timed with CUDA events on its stream after construction and warm-up,
  ``e2e`` the same whole job as ours with the same bytes declared.
Multi-GPU: the single network does not shard; ``--gpus N`` runs N
independent replicas (one per rank, distinct seeds), weak scaling.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

DT = 0.05
WORKLOAD = dict(N=1_000_000, k=32, p=0.1, max_delay=64)
WORKLOAD_NAME = ("plain engine at scale: Watts-Strogatz N=1e6, k=32, p=0.1, "
                 "delays U[1,64], dt=0.05, controller on")


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, local):
    import torch

    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=600))


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist

        if torch.cuda.is_available():
            dist.barrier(device_ids=[torch.cuda.current_device()])
        else:
            dist.barrier()


def max_over_ranks(x, world):
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel="step_kernel"):
    """DRAM bytes per launch of ``kernel`` on this workload from the
    committed ncu summary (profiles/<kernel>_traffic.txt), or None."""
    path = os.path.join(REPO, "profiles", f"{kernel}_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = f"/tmp/lev_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), max=float(parts[2]),
                                 power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        load = [r for r in rows if r["power"] > 250.0] or rows
        reasons = set()
        for r in load:
            for k, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                            ("swt", "sw_thermal_slowdown"), ("swp", "sw_power_cap")):
                if r[k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in load),
                "sm_max_mhz": max(r["max"] for r in rows),
                "reasons": sorted(reasons), "samples": len(load)}


def build_workload(seed):
    from leviathan_v1_b200.graphs import make_network

    return make_network(WORKLOAD["N"], WORKLOAD["k"], WORKLOAD["p"],
                        WORKLOAD["max_delay"], seed)


def bench_config(N, E):
    """The workload description both arms print (identical dicts)."""
    return {"workload": WORKLOAD_NAME, "N": N, "E": E,
            "max_delay": WORKLOAD["max_delay"], "dt": DT,
            "parallelism": "replicas (one network per GPU; a single network "
                           "does not shard)",
            "l2": "inputs (1.2 GB) larger than L2 (126 MB); no flush"}


def h2d_bytes(N, E):
    """Host->device bytes of one job: row_ptr, col_idx, delays, weights,
    theta, theta_hat, omega."""
    return (N + 1) * 4 + E * (4 + 1 + 4) + N * 4 * 3


def d2h_bytes(N, K):
    """Device->host bytes of one job: r of every step, final phases."""
    return 4 * K + 4 * N


def launches_per_job(K, pairs, block=256):
    """Kernel launches of K steps run as step blocks of `block` steps (one
    graph each): a reset of the r-history counter per block, then per two
    steps pair_kernel, reduce_kernel, finish_kernel, reduce_kernel -- or one
    step_kernel per step."""
    n = 0
    for b0 in range(0, K, block):
        L = min(block, K - b0)
        n += 1 + ((L // 2) * 4 + (L % 2) if pairs else L)
    return n


def algorithmic_bytes(N, E):
    """Bytes one step must move (reference layout): per edge col 4 + delay 1
    + weight read 4 + weight write 4 + delayed-phase gather 4 = 17; per node
    row_ptr 4 + theta r/w 8 + theta_hat r/w 8 + omega 4 + omega_hat r/w 8 +
    ring-slot write 4 = 36; plus row_ptr[N]."""
    return 17 * E + 36 * N + 4


def _phase_errors(theta, theta64, r, r64):
    from oracle64 import circular_distance

    d = circular_distance(theta, theta64)
    return {"max_wrapped_phase_rad": float(d.max()), "mean_wrapped_phase_rad": float(d.mean()),
            "max_abs_r": float(np.abs(np.asarray(r, np.float64) - np.asarray(r64)).max())}


def cpu_baseline_and_fp64_prefix(net, budget_s=20.0):
    """FP64 NumPy oracle (oracle/oracle64.py) on the host over the first
    steps of the bench network, as many as fit in about ``budget_s``
    (at least 3): timed, it is the CPU baseline; its phases after those
    steps, against the engine's after the same steps (both math modes),
    state the FP64 error of the bench configuration over that prefix."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from oracle64 import OracleEngine

    from leviathan_v1_b200 import LeviathanEngine

    o = OracleEngine(*net.engine_args())
    t0 = time.perf_counter()
    r64 = [o.step(DT)]
    first = time.perf_counter() - t0
    n = max(3, min(50, int(budget_s / max(first, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(n - 1):
        r64.append(o.step(DT))
    el = time.perf_counter() - t0
    base = {"value": net.E * (n - 1) / el, "unit": "edge-updates/s", "cores": 1,
            "kind": "port",
            "sample": f"steps 2..{n} of the bench network (step 1 untimed), FP64 "
                      f"NumPy oracle, single-threaded NumPy, {os.cpu_count()} host "
                      f"cores present"}
    errs = {"steps": n, "note": f"prefix of the run: the first {n} steps from the "
                                f"bench's initial state"}
    for mode in ("reference", "accurate"):
        e = LeviathanEngine(*net.engine_args(), math_mode=mode)
        r = e.step_n(DT, n)
        errs[mode] = _phase_errors(e.get_theta(), o.theta, r, r64)
        e.close()
    return base, errs


def fp64_error_batched_prefix(eng, nets, params, picks, steps=10):
    """Error of sampled networks of a batched engine against the FP64
    oracle over the next ``steps`` steps from the engine's current state
    (a prefix; the engine must be at its initial state)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from oracle64 import OracleEngine

    r = eng.step_n(DT, steps)
    out = {"steps": steps, "networks": []}
    for i in picks:
        o = OracleEngine(*nets[i].engine_args(), params=params[i])
        r64 = o.run(DT, steps)
        err = _phase_errors(eng.get_theta(i), o.theta, r[:, i], r64)
        err.update(N=nets[i].N, E=nets[i].E, K=params[i]["g"])
        out["networks"].append(err)
    out["max_wrapped_phase_rad"] = max(x["max_wrapped_phase_rad"] for x in out["networks"])
    return out


def fp64_error_small():
    """Wrapped-phase error after 200 steps against the FP64 oracle on the
    small configuration (N=1000, k=20), both math modes."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from oracle64 import OracleEngine, circular_distance

    from leviathan_v1_b200 import LeviathanEngine
    from leviathan_v1_b200.graphs import config_small

    net = config_small(0)
    o = OracleEngine(*net.engine_args())
    o.run(DT, 200)
    out = {}
    for mode in ("reference", "accurate"):
        e = LeviathanEngine(*net.engine_args(), math_mode=mode)
        e.step_n(DT, 200)
        out[mode] = float(circular_distance(e.get_theta(), o.theta).max())
        e.close()
    return out


# ---------------------------------------------------------------------------
# plain engine, small (N=1000, k=20): latency-bound, reported in us/step
# ---------------------------------------------------------------------------
def _resident_run(net, steps, label):
    """Steps of a network small enough for the cluster- or grid-resident
    paths (autotuned against graph replay), CUDA events on the engine
    stream.  Its working set is L2-resident, so the achieved figure is the
    algorithmic bytes per step (17E + 36N + 4) over the step time, against L2
    rather than HBM."""
    import torch

    from leviathan_v1_b200 import LeviathanEngine

    e = LeviathanEngine(*net.engine_args())
    e.autotune(DT, trial_steps=10)  # cluster, grid or graph replay
    ci, gi = e.cluster_info(), e.grid_info()
    stream = torch.cuda.ExternalStream(e.stream_ptr)
    e.step_n_async(DT, steps)  # issued directly
    e.step_n_async(DT, steps)  # records the graph the timed block replays
    e.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    e.step_n_async(DT, steps)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    e.close()
    if ci["enabled"]:
        path = "cluster-resident kernel, %d CTAs" % ci["ctas"]
    elif gi["enabled"]:
        path = "grid-resident kernel, %d CTAs of %d rows" % (gi["ctas"], gi["rows_per_cta"])
    else:
        path = "step kernel graph replay"
    alg = algorithmic_bytes(net.N, net.E)
    step_s = ms / 1e3 / steps
    return {"workload": label, "N": net.N, "E": net.E, "steps": steps,
            "us_per_step": step_s * 1e6, "edge_updates_per_s": net.E / step_s,
            "algorithmic_bytes_per_step": alg, "algorithmic_GBps": alg / step_s / 1e9,
            "path": path}


def run_small(args):
    from leviathan_v1_b200.graphs import config_small

    return _resident_run(config_small(0), 500, "Watts-Strogatz N=1000, k=20, p=0.1, "
                         "delays U[1,50], 500 steps, controller on")


def run_mid(args):
    from leviathan_v1_b200.graphs import config_adjoint

    return _resident_run(config_adjoint(0), 2000, "Watts-Strogatz N=1e4, k=20, p=0.1, "
                         "delays U[1,50], 2000 steps, controller on (the adjoint "
                         "configuration's plain engine, reference math)")


# ---------------------------------------------------------------------------
# batched sweep (512 networks, one launch per step, sharded over ranks)
# ---------------------------------------------------------------------------
def run_batched(args, rank, world, plain_value):
    import torch

    from leviathan_v1_b200 import BatchEngine, LeviathanEngine
    from leviathan_v1_b200.graphs import batch_specs, build_batch
    from leviathan_v1_b200.sharding import gather_results, shard_by_edges, summarize_r

    specs = batch_specs(512, seed=0)
    shards = shard_by_edges([s["E"] for s in specs], world)
    mine = shards[rank]
    nets, params = build_batch([specs[i] for i in mine])
    E_local = sum(n.E for n in nets)
    N_local = sum(n.N for n in nets)
    eng = BatchEngine([n.as_dict() for n in nets], params=params)
    tune = eng.autotune(DT, trial_steps=5)  # the state is restored afterwards
    pair_info = eng.pair_info()
    # FP64 error over a 10-step prefix of four sampled networks (K spread),
    # from the initial state; the timing below continues from there
    picks = [i for i in np.argsort([p["g"] for p in params])[[0, len(nets) // 3,
                                                              2 * len(nets) // 3, -1]]]
    picks = [int(i) for i in picks if nets[i].N <= 20_000] or [int(np.argmin([n.N for n in nets]))]
    fp64 = fp64_error_batched_prefix(eng, nets, params, picks) if rank == 0 else None
    if rank != 0:
        eng.step_n(DT, 10)
    S = args.batched_steps
    eng.step_n_async(DT, max(args.warmup, 3))
    eng.step_n_async(DT, S)
    eng.step_n_async(DT, S)  # records the graph the timed block replays
    eng.synchronize()
    stream = torch.cuda.ExternalStream(eng.stream_ptr)
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    eng.step_n_async(DT, S)
    ev1.record(stream)
    ev1.synchronize()
    barrier(world)
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    E_tot = sum_over_ranks(E_local, world)
    N_tot = sum_over_ranks(N_local, world)
    value = E_tot * S / (ms / 1e3)
    # r(K) curve: sweep continues to 1000 steps in total, mean r of the last 100
    done = 10 + max(args.warmup, 3) + 3 * S
    r = eng.step_n(DT, max(1000 - done, 100))
    curve = gather_results(mine, summarize_r(r, 100), len(specs))
    eng.close()
    # the same networks one engine at a time (the reference's serial pattern,
    # experiments/phase_sweep.py), a sample of 16 networks on this rank
    sample = nets[:: max(1, len(nets) // 16)][:16]
    t0 = time.perf_counter()
    E_s = 0
    for n, p in zip(sample, params[:: max(1, len(nets) // 16)][:16]):
        e = LeviathanEngine(*n.engine_args(), params=p)
        e.step_n(DT, 50)
        E_s += n.E * 50
        e.close()
    serial = E_s / (time.perf_counter() - t0)
    bins = np.linspace(0, 4, 9)
    Ks = np.array([s["K"] for s in specs])
    r_of_K = [float(np.nanmean(curve[(Ks >= lo) & (Ks < hi + (hi == 4)), 0]))
              for lo, hi in zip(bins[:-1], bins[1:])]
    return {"networks": len(specs), "nodes": int(N_tot), "edges": int(E_tot),
            "steps": S, "ms_per_step": ms / S, "edge_updates_per_s": value,
            "vs_plain_kernel": value / plain_value if plain_value else None,
            "serial_engines_edge_updates_per_s": serial,
            "serial_engines_note": "16 sampled networks, one engine each, 50 steps "
                                   "per call incl. engine construction",
            "autotune": {"chosen": tune["chosen"], "ms": tune["ms"],
                         "variants": tune["variants"], "pairs": pair_info},
            "r_of_K_bins_0_to_4": r_of_K,
            "fp64_error_prefix": fp64,
            "algorithmic_bytes_per_step": int(17 * E_tot + 36 * N_tot)}


# ---------------------------------------------------------------------------
# adjoint (N=1e4, k=20, 2000 steps, checkpoint every 50) and differentiable
# reservoir (batch 64 x N=5e4, k=20, 1000 steps)
# ---------------------------------------------------------------------------
def _cuda_time(fn):
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    return out, time.perf_counter() - t0


def run_adjoint(args):
    import torch

    from leviathan_v1_b200 import LeviathanEngine
    from leviathan_v1_b200.adjoint import Adjoint, simulate
    from leviathan_v1_b200.graphs import config_adjoint

    T, C = args.adjoint_steps, 50
    net = config_adjoint(0)
    eng = LeviathanEngine(*net.engine_args(), math_mode="accurate")
    adj = Adjoint(eng, segment=C, max_steps=T)
    om = torch.tensor(net.omega, device="cuda", requires_grad=True)
    w0 = torch.tensor(net.weights, device="cuda", requires_grad=True)
    K = torch.full((1,), 1.5, device="cuda", requires_grad=True)
    t = torch.arange(1, T + 1, device="cuda", dtype=torch.float32)
    tgt = 0.5 + 0.2 * torch.sin(2 * math.pi * t / 400.0)

    def fwd():
        return simulate(adj, om, w0, K, T, DT)[:, 0]

    def fwd_bwd():
        r = fwd()
        L = torch.mean((r - tgt) ** 2)
        L.backward()
        return L

    fwd_bwd()  # warm-up
    om.grad = w0.grad = K.grad = None
    _, t_f = _cuda_time(fwd)
    L, t_fb = _cuda_time(fwd_bwd)
    plain = LeviathanEngine(*net.engine_args(), math_mode="accurate")
    plain.step_n(DT, 50)
    _, t_plain = _cuda_time(lambda: plain.step_n(DT, T))
    plain.close()
    out = {"workload": "N=1e4, k=20, delays U[1,50], T=2000 steps, checkpoint every 50, "
                       "loss = MSE(r, 0.5 + 0.2 sin(2 pi t/400)), grads w.r.t. omega, w, K",
           "N": net.N, "E": net.E, "T": T, "segment": C,
           "fwd_s": t_f, "fwd_bwd_s": t_fb, "fwd_bwd_over_fwd": t_fb / t_f,
           "fwd_edge_updates_per_s": net.E * T / t_f,
           "plain_engine_edge_updates_per_s": net.E * T / t_plain,
           "loss": float(L.detach()), "grad_norms": {
               "omega": float(om.grad.norm()), "w": float(w0.grad.norm()),
               "K": float(K.grad.abs().sum())},
           "device_bytes": adj.device_bytes,
           "gradient_check": "rel. error <= 1e-3 vs FP64 autograd and FP64 finite "
                             "differences at N=200, k=8, 100 steps (tests/test_adjoint_gpu.py)"}
    adj.close()
    eng.close()
    return out


def run_reservoir(args):
    import torch

    from leviathan_v1_b200.graphs import config_reservoir
    from leviathan_v1_b200.reservoir import DifferentiableReservoir, make_inputs

    B, T = 64, args.reservoir_steps
    net = config_reservoir(0)
    model = DifferentiableReservoir(net, B, n_input=256, T=T, segment=50, seed=0)
    x = torch.tensor(make_inputs(B, T, seed=0), device="cuda")

    def fwd():
        with torch.no_grad():
            return model(x, DT)

    def fwd_bwd():
        y, r = model(x, DT)
        L = model.loss(y, x, 10)
        L.backward()
        return L

    fwd_bwd()  # warm-up
    model.zero_grad()
    _, t_f = _cuda_time(fwd)
    L, t_fb = _cuda_time(fwd_bwd)
    E_tot = net.E * B
    out = {"workload": "batch 64 x (N=5e4, k=20, delays U[1,50]), T=1000, 256 input nodes, "
                       "readout on cos/sin of all phases predicts x(t+10); grads w.r.t. W_in, "
                       "omega, readout",
           "batch": B, "N": net.N, "E_per_copy": net.E, "T": T,
           "fwd_s": t_f, "fwd_bwd_s": t_fb, "fwd_bwd_over_fwd": t_fb / t_f,
           "fwd_edge_updates_per_s": E_tot * T / t_f,
           "loss": float(L.detach()),
           "grad_norms": {"w_in": float(model.w_in.grad.norm()),
                          "omega": float(model.omega.grad.norm()),
                          "readout": float(model.read_a.grad.norm() + model.read_b.grad.norm())},
           "device_bytes": model.adj.device_bytes,
           "gradient_check": "rel. error <= 1e-3 vs FP64 autograd at N=200, batch 3, 60 "
                             "steps (tests/test_reservoir_gpu.py)"}
    model.close()
    return out


# ---------------------------------------------------------------------------
# our engine
# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local):
    import torch

    from leviathan_v1_b200 import LeviathanEngine

    net = build_workload(seed=rank)
    N, E = net.N, net.E
    K, W = args.steps, args.warmup

    eng = LeviathanEngine(*net.engine_args())
    # the in-project autotuner picks the step-kernel variant for this degree
    # distribution (state is restored; later engines of the process reuse it)
    tune = eng.autotune(DT, trial_steps=10)
    cls = next(t["cls"] for t in eng.tuning() if t["tiles"])
    pair_info = eng.pair_info()[cls]
    stream = torch.cuda.ExternalStream(eng.stream_ptr)
    sampler = ClockSampler(torch.cuda.current_device()).start()

    # warm-up: the first block of a length is issued directly, the second
    # records the graph that the timed block replays
    eng.step_n_async(DT, W)
    eng.step_n_async(DT, K)
    eng.step_n_async(DT, K)
    eng.synchronize()

    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    eng.step_n_async(DT, K)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    ms_max = max_over_ranks(ms, world)
    edges_total = sum_over_ranks(E, world)
    value = edges_total * K / (ms_max / 1e3)
    r_last = eng.get_r()
    # launch durations of the dominant kernel (CUDA events on the engine
    # stream; pair_kernel, then finish_kernel, of a two-step round)
    t_launch = eng.time_launches(DT, 20)
    eng.close()

    # end-to-end through the public API with host buffers: construction from
    # host arrays, K steps with r of every step returned to the host (the
    # block form used by LeviathanObservatory.run_baseline), final phases
    h2d = h2d_bytes(N, E)
    d2h = d2h_bytes(N, K)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2 = LeviathanEngine(*net.engine_args())
    t1 = time.perf_counter()
    r_hist = e2.step_n(DT, K)
    t2 = time.perf_counter()
    theta = e2.get_theta()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_parts = {"construct_s": t1 - t0, "step_n_s": t2 - t1,
                 "get_theta_s": e2e_s - (t2 - t0),
                 "construct_ms_by_phase": e2.create_profile(),
                 "h2d_GBps_of_construct": h2d_bytes(N, E) / (t1 - t0) / 1e9}
    e2.close()
    e2e_s = max_over_ranks(e2e_s, world)
    # the same job with one step(dt) call per step (reference call pattern)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e3 = LeviathanEngine(*net.engine_args())
    for _ in range(K):
        e3.step(DT)
    e3.get_theta()
    torch.cuda.synchronize()
    e3_s = max_over_ranks(time.perf_counter() - t0, world)
    e3.close()
    e2e = {"value": edges_total * K / e2e_s, "unit": "edge-updates/s",
           "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
           "path": "LeviathanEngine(host arrays) + step_n(dt, K) -> r[K] + get_theta()",
           "seconds": e2e_s, "parts": e2e_parts,
           "per_step_calls": {"value": edges_total * K / e3_s, "seconds": e3_s,
                              "path": "LeviathanEngine(host arrays) + K x step(dt) -> r "
                                      "+ get_theta()"}}

    step_s = ms / 1e3 / K
    alg = algorithmic_bytes(N, E)
    peak, peak_kind = measured_peaks()
    pairs = pair_info["enabled"] and pair_info["pair_variant"] >= 0
    if pairs:
        # pair_kernel: two steps' edge work, 2 x 17 B per edge; per node
        # row_ptr 4, theta r/w 8, theta_hat r/w 8, omega_hat r/w 8, omega 4,
        # ring write 4, parked (sum, eps) write 8 = 44 B
        kernel = "lev::pair_kernel (steps t and t+1 but the last integrate)"
        alg_launch = 34 * E + 44 * N + 4
        launch_s = t_launch[0] / 1e3
        traffic = profiled_traffic("pair_kernel")
    else:
        kernel = "lev::step_kernel"
        alg_launch = alg
        launch_s = t_launch[0] / 1e3
        traffic = profiled_traffic("step_kernel")
    achieved = alg_launch / launch_s / 1e9
    line = {
        "metric": "edge-updates/s", "value": value, "unit": "edge-updates/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms_max / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Watts-Strogatz, seeded states)",
        "config": bench_config(N, E),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "kernel": kernel,
                     "algorithmic_bytes_per_launch": alg_launch,
                     "launch_us": t_launch[0] * 1e3,
                     "second_launch_us": t_launch[1] * 1e3,
                     "step_sequence": {"algorithmic_bytes_per_step": alg,
                                       "achieved": alg / step_s / 1e9,
                                       "frac": alg / step_s / 1e9 / peak},
                     "one_step_variant": tune["variants"][tune["chosen"][cls]],
                     "two_steps_per_launch": pair_info},
        "e2e": e2e,
        "gpu_launches": launches_per_job(K, pairs),
        "clocks": clocks,
        "r_final": r_last,
        "theta_finite": bool(np.all(np.isfinite(theta))),
    }
    if not args.no_batched:
        line["batched"] = run_batched(args, rank, world, value)
    if rank == 0:
        line["small"] = run_small(args)
        line["mid"] = run_mid(args)
    if rank == 0 and not args.no_adjoint:
        line["adjoint"] = run_adjoint(args)
        line["reservoir"] = run_reservoir(args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], line["fp64_error_prefix"] = cpu_baseline_and_fp64_prefix(
            net, budget_s=args.cpu_budget)
    if rank == 0 and not args.no_fp64_check:
        line["fp64_error_small_200_steps"] = fp64_error_small()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# reference engine (oracle/_ref, built from the reference sources)
# ---------------------------------------------------------------------------
def run_reference(args, rank, world, local):
    """The reference engine, same network, same job, same GPU.

    ``value``: after construction and W warm-up steps, K ``leviathan_step``
    calls (each with its stock 4-byte r read-back, stream synchronisation and
    host gain controller, leviathan_kernel.cu:391-438) timed with CUDA events
    on the engine's own stream.  ``e2e``: construction from host arrays
    (leviathan_init, :270-389), K steps and ``leviathan_get_theta`` (:440),
    wall clock, with the host<->device bytes declared exactly as for this
    repository's arm.  Each metric comes from the faster of the two
    reference builds at it."""
    if rank != 0:
        return
    import torch

    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import refengine

    net = build_workload(seed=0)
    N, E = net.N, net.E
    K, W = args.steps, args.warmup
    device, e2e_s, parts = {}, {}, {}
    for flavor in ("sm100a", "stock"):
        if not refengine.available(flavor):
            continue
        ref = refengine.RefEngine(*net.engine_args(), flavor=flavor)
        for _ in range(W):
            ref.step(DT)
        stream = torch.cuda.ExternalStream(ref.stream)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(K):
            ref.step(DT)
        ev1.record(stream)
        ev1.synchronize()
        device[flavor] = E * K / (ev0.elapsed_time(ev1) / 1e3)
        ref.close()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ref = refengine.RefEngine(*net.engine_args(), flavor=flavor)
        t1 = time.perf_counter()
        for _ in range(K):
            ref.step(DT)
        t2 = time.perf_counter()
        ref.get_theta()
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        parts[flavor] = {"construct_s": t1 - t0, "steps_s": t2 - t1,
                         "get_theta_s": el - (t2 - t0)}
        ref.close()
        e2e_s[flavor] = el
    if not device:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref reference build missing (make -C oracle)"}))
        return
    best = max(device, key=device.get)
    v = device[best]
    best_e2e = min(e2e_s, key=e2e_s.get)  # each metric from the build that is faster at it
    line = {
        "impl": "reference", "metric": "edge-updates/s", "value": v,
        "unit": "edge-updates/s", "n_gpus": 1, "steps": K, "warmup": W,
        "ms_per_step": E / v * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Watts-Strogatz, seeded states)",
        "config": bench_config(N, E),
        "timing": "value: CUDA events on the reference engine's stream around K "
                  "leviathan_step calls after construction and W warm-up steps",
        "reference_builds": {"device": device, "e2e_seconds": e2e_s},
        "reference_build_used": best, "reference_build_used_e2e": best_e2e,
        "e2e": {"value": E * K / e2e_s[best_e2e], "unit": "edge-updates/s",
                "h2d_bytes_per_step": h2d_bytes(N, E) / K,
                "d2h_bytes_per_step": d2h_bytes(N, K) / K,
                "path": "leviathan_init(host arrays) + K x leviathan_step -> r "
                        "+ leviathan_get_theta",
                "seconds": e2e_s[best_e2e], "parts": parts[best_e2e]},
        "gpu_launches": 4 * K,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-check", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    ap.add_argument("--reservoir-steps", type=int, default=1000)
    ap.add_argument("--batched-steps", type=int, default=200)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_env()
    init_dist(world, local)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
