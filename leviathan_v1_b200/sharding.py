"""Multi-GPU execution of batched sweeps.

Networks of a sweep are independent, so the sweep shards by whole networks:
each rank (one process per GPU) runs a ``BatchEngine`` over its share, with
no collective inside the step loop; per-network results are gathered once at
the end.  Shares are balanced by edge count (the step is bandwidth-bound and
its cost is proportional to edges).  A single network is never split: at the
sizes of this path it fits one GPU many times over, so more GPUs run more
networks (or replicas), not bigger ones.
"""

from __future__ import annotations

import heapq
from typing import Sequence

import numpy as np


def shard_by_edges(edge_counts: Sequence[int], world_size: int) -> list:
    """Greedy longest-processing-time assignment of networks to ranks.

    Returns ``world_size`` lists of network indices (each sorted); every
    network appears exactly once; deterministic for equal inputs."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(edge_counts)), key=lambda i: (-int(edge_counts[i]), i))
    heap = [(0, r) for r in range(world_size)]
    heapq.heapify(heap)
    shards = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(edge_counts[i]), r))
    return [sorted(s) for s in shards]


def summarize_r(r_hist: np.ndarray, tail: int) -> np.ndarray:
    """Per-network (mean, std) of r over the last ``tail`` steps;
    ``r_hist`` is [steps, nets]."""
    t = r_hist[-tail:] if tail > 0 else r_hist
    return np.stack([t.mean(axis=0), t.std(axis=0)], axis=1)


def gather_results(local_indices: Sequence[int], local_values: np.ndarray,
                   total: int, group=None) -> np.ndarray:
    """Assemble per-network rows computed on every rank into one
    ``[total, ...]`` array, available on every rank (all_gather of Python
    objects: one call after the sweep, not per step)."""
    import torch.distributed as dist

    payload = (list(map(int, local_indices)), np.asarray(local_values))
    if dist.is_available() and dist.is_initialized():
        objs = [None] * dist.get_world_size(group)
        dist.all_gather_object(objs, payload, group=group)
    else:
        objs = [payload]
    shape = None
    for idx, vals in objs:
        if len(idx):
            shape = vals.shape[1:]
            break
    out = np.full((total,) + (shape or ()), np.nan)
    for idx, vals in objs:
        for i, v in zip(idx, vals):
            out[i] = v
    return out


def run_sweep(specs, steps: int, dt: float = 0.05, tail: int = 100,
              rank: int = 0, world_size: int = 1, autotune: bool = True,
              math_mode: str = "reference", engine_factory=None) -> np.ndarray:
    """r(K) sweep over ``specs`` (see ``graphs.batch_specs``) sharded over
    ``world_size`` ranks; returns [len(specs), 2] (mean, std of r over the
    last ``tail`` steps) on every rank.  ``engine_factory(nets, params,
    math_mode)`` builds a rank's engine (default: a ``BatchEngine``; tests
    substitute a host stand-in to run the sharding on CPU ranks)."""
    from .graphs import build_batch

    if engine_factory is None:
        from .engine import BatchEngine

        def engine_factory(nets, params, math_mode):
            return BatchEngine([n.as_dict() for n in nets], params=params,
                               math_mode=math_mode)

    shards = shard_by_edges([s["E"] for s in specs], world_size)
    mine = shards[rank]
    if mine:
        nets, params = build_batch([specs[i] for i in mine])
        eng = engine_factory(nets, params, math_mode)
        if autotune:
            eng.autotune(dt)
        r = eng.step_n(dt, steps)
        eng.close()
        local = summarize_r(r, tail)
    else:
        local = np.zeros((0, 2))
    return gather_results(mine, local, len(specs))
