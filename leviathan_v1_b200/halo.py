"""One network split over several GPUs: the halo engine.

Replaces the reference's multi-GPU path, which does not work: its halo
pack/unpack kernels are never launched (leviathan_multigpu.cu:97-115), its
step runs every GPU's engine one after the other and averages the per-GPU
|r| on the host (:218-238), and its partitioner drops every edge that crosses
a partition boundary (python/partition.py:121).  Here every edge is kept and
a partitioned run is the single-GPU run, bit for bit.

Design (one process per GPU, ``torch.distributed`` for the plumbing):

* **Partition.** The N rows are cut into contiguous ranges of whole 256-row
  tiles, ``C = ceil(ceil(N / 256) / world)`` tiles per rank (the last rank
  takes the rest).  Contiguous ranges keep the Watts-Strogatz ring lattice
  local; only the rewired edges and the range ends reach other ranks.
* **Halo.** A rank's rows read the phases of some nodes other ranks own.
  Those nodes get ring columns after the rank's own columns, so every
  delayed gather stays a local ring read; each step the owners send
  theta(t+1) of exactly those nodes, which lands in the ring slot of
  theta(t+1) before the next step reads it.
* **Order parameter.** Each rank writes the (sum cos, sum sin) partials of
  its tiles at their global tile positions; an all-gather of the partials
  (8 bytes per 256 nodes) gives every rank the same array, reduced in the
  reference's order (leviathan_kernel.cu:242-263) -- so r and the gain g of
  the controller (:431-435) are identical on every rank and equal to the
  single-GPU engine's.  The all-gather replaces the reference's host mean.
* **Per step:** local step (one launch) -> all-gather of tile partials ->
  r and g (one launch) -> pack -> send/recv -> unpack.  All on the engine
  stream; the collectives run on it through ``torch.cuda.ExternalStream``.

The device work is the C ABI ``lev_part_*`` (``include/leviathan_b200.h``).
The ``core`` argument of :class:`PartitionedEngine` is a test seam for the
per-rank compute (the package itself has only the CUDA core).
"""

from __future__ import annotations

import contextlib
import ctypes as C
import threading
from dataclasses import dataclass, field

import numpy as np

TILE = 256


# ---------------------------------------------------------------------------
# partition plan (host only)
# ---------------------------------------------------------------------------
@dataclass
class RankPlan:
    """What one rank owns, reads and exchanges."""

    rank: int
    world: int
    row0: int                  # first own global row (multiple of 256)
    row1: int                  # one past the last own row
    tile_off: int              # first global tile
    tiles_per_rank: int        # C: all-gather chunk of every rank, in tiles
    ntiles_global: int
    N_global: int
    row_ptr: np.ndarray        # local CSR of the own rows
    col_idx: np.ndarray        # renumbered: own j -> j - row0, halo -> N + position
    edge0: int                 # first global edge (CSR order) of the own rows
    edge1: int
    halo: np.ndarray           # global ids of the halo nodes, sorted
    recv: dict = field(default_factory=dict)  # peer -> positions in ``halo`` (contiguous)
    send: dict = field(default_factory=dict)  # peer -> own local node indices

    @property
    def N(self) -> int:
        return self.row1 - self.row0

    @property
    def n_halo(self) -> int:
        return int(self.halo.size)


class PartitionPlan:
    """Contiguous tile-aligned row ranges and the halo lists of every rank.

    Built from the whole network's CSR, which every rank holds (the graph is
    generated from a seed on every rank), so no request lists need to be
    exchanged: what peer p receives from rank q is p's halo restricted to
    q's rows, in global id order on both sides."""

    def __init__(self, row_ptr, col_idx, world: int):
        rp = np.asarray(row_ptr, dtype=np.int64)
        col = np.asarray(col_idx, dtype=np.int64)
        N = rp.size - 1
        if world < 1:
            raise ValueError("world must be >= 1")
        T = -(-N // TILE)
        C_ = -(-T // world)
        if (world - 1) * C_ >= T:
            raise ValueError(f"{N} nodes ({T} tiles of {TILE}) are too few for "
                             f"{world} partitions of whole tiles")
        self.N, self.world, self.ntiles, self.tiles_per_rank = N, world, T, C_
        self.bounds = [(min(r * C_ * TILE, N), min((r + 1) * C_ * TILE, N))
                       for r in range(world)]
        starts = np.array([b[0] for b in self.bounds] + [N], dtype=np.int64)
        self.ranks = []
        for r, (row0, row1) in enumerate(self.bounds):
            e0, e1 = int(rp[row0]), int(rp[row1])
            cols = col[e0:e1]
            own = (cols >= row0) & (cols < row1)
            halo = np.unique(cols[~own])
            local = np.empty(cols.size, dtype=np.int32)
            local[own] = (cols[own] - row0).astype(np.int32)
            local[~own] = (row1 - row0 + np.searchsorted(halo, cols[~own])).astype(np.int32)
            owner = np.searchsorted(starts, halo, side="right") - 1
            recv = {}
            for p in range(world):
                if p == r:
                    continue
                pos = np.flatnonzero(owner == p)
                if pos.size:
                    recv[p] = pos.astype(np.int32)
            self.ranks.append(RankPlan(
                rank=r, world=world, row0=row0, row1=row1, tile_off=r * C_,
                tiles_per_rank=C_, ntiles_global=T, N_global=N,
                row_ptr=(rp[row0:row1 + 1] - e0).astype(np.int32), col_idx=local,
                edge0=e0, edge1=e1, halo=halo, recv=recv))
        # what each rank sends: the receiver's halo nodes in the sender's rows
        for p, rpl in enumerate(self.ranks):
            for q, pos in rpl.recv.items():
                snd = self.ranks[q]
                snd.send[p] = (rpl.halo[pos] - snd.row0).astype(np.int32)

    def rank(self, r: int) -> RankPlan:
        return self.ranks[r]

    def halo_bytes_per_step(self) -> int:
        """theta(t+1) bytes that cross between ranks per step (all ranks)."""
        return 4 * sum(int(p.n_halo) for p in self.ranks)


# ---------------------------------------------------------------------------
# exchanges
# ---------------------------------------------------------------------------
class DistExchange:
    """Collectives of the halo step over ``torch.distributed`` (NCCL between
    GPUs, gloo on the CPU).  ``stream`` (a ``torch.cuda.Stream``) is the
    engine stream the collectives are ordered on."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nccl = dist.get_backend(group) == "nccl"

    def _on(self, stream):
        if stream is None:
            return contextlib.nullcontext()
        import torch

        return torch.cuda.stream(stream)

    def allgather(self, out, chunk, stream=None):
        """``out`` [world * C, ...] := every rank's ``chunk`` [C, ...] in rank
        order (this rank's own chunk may be a view of ``out``)."""
        n = chunk.numel()
        own = out.view(-1)[self.rank * n:(self.rank + 1) * n]
        in_place = own.data_ptr() == chunk.data_ptr()
        if self.world == 1:
            if not in_place:
                own.copy_(chunk.view(-1))
            return
        with self._on(stream):
            if self.nccl:
                # one collective into `out`; NCCL takes the rank's own slot of
                # the output as the input (its in-place all-gather)
                self.dist.all_gather_into_tensor(out.view(-1), own if in_place else
                                                 chunk.reshape(-1), group=self.group)
            else:
                parts = list(out.view(self.world, *chunk.shape).unbind(0))
                self.dist.all_gather(parts, chunk.clone(), group=self.group)

    def exchange(self, sends: dict, recvs: dict, stream=None):
        """Point-to-point: ``sends[peer]`` goes to peer, ``recvs[peer]`` is
        filled from peer."""
        ops = []
        P2P = self.dist.P2POp
        # a fixed order (by peer) on every rank: sends and receives of a
        # pair are matched the same way everywhere
        for peer in sorted(set(sends) | set(recvs)):
            if peer in sends:
                ops.append(P2P(self.dist.isend, sends[peer], peer, self.group))
            if peer in recvs:
                ops.append(P2P(self.dist.irecv, recvs[peer], peer, self.group))
        if not ops:
            return
        with self._on(stream):
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()


class ThreadExchange:
    """All partitions of a network in one process, one thread per rank (for
    several GPUs driven from one process, or several partitions on one GPU).
    Each rank's collective calls meet at a barrier; buffers are exchanged by
    copies after every producer's stream has finished."""

    def __init__(self, world: int):
        self.world = world
        self._bar = threading.Barrier(world)
        self._slots: dict = {}

    def bind(self, rank: int) -> "_ThreadRank":
        return _ThreadRank(self, rank)


class _ThreadRank:
    def __init__(self, hub: ThreadExchange, rank: int):
        self.hub, self.rank, self.world = hub, rank, hub.world

    @staticmethod
    def _sync(stream):
        if stream is not None:
            stream.synchronize()

    def allgather(self, out, chunk, stream=None):
        import torch

        self._sync(stream)
        self.hub._slots[("ag", self.rank)] = chunk
        self.hub._bar.wait()
        parts = out.view(self.world, *chunk.shape)
        with (torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()):
            for q in range(self.world):
                src = self.hub._slots[("ag", q)]
                if src.data_ptr() != parts[q].data_ptr():
                    parts[q].copy_(src)
        self._sync(stream)
        self.hub._bar.wait()

    def exchange(self, sends: dict, recvs: dict, stream=None):
        import torch

        self._sync(stream)
        for peer, t in sends.items():
            self.hub._slots[("p2p", self.rank, peer)] = t
        self.hub._bar.wait()
        with (torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()):
            for peer, buf in recvs.items():
                buf.copy_(self.hub._slots[("p2p", peer, self.rank)])
        self._sync(stream)
        self.hub._bar.wait()


# ---------------------------------------------------------------------------
# per-rank compute: the CUDA partition engine
# ---------------------------------------------------------------------------
class CudaPartition:
    """``lev_part_*`` engine of one rank on the current CUDA device."""

    def __init__(self, plan: RankPlan, delays, weights, theta, theta_hat, omega,
                 theta_halo, max_delay, params=None, math_mode=0):
        import torch

        from . import _lib
        from ._lib import check

        self._lib, self._check = _lib.load(), check
        f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
        keep = [np.ascontiguousarray(plan.row_ptr, np.int32),
                np.ascontiguousarray(plan.col_idx, np.int32),
                np.ascontiguousarray(delays, np.uint8), f32(weights), f32(theta),
                f32(theta_hat), f32(omega), f32(theta_halo)]
        ptr = lambda a: C.c_void_p(a.ctypes.data) if a.size else C.c_void_p(0)
        p = _lib.make_params(**(params or {}))
        h = C.c_void_p()
        check(self._lib.lev_part_create(
            C.byref(h), plan.N, plan.n_halo, int(max_delay), *[ptr(a) for a in keep],
            plan.N_global, plan.tile_off, plan.ntiles_global, C.byref(p), int(math_mode)))
        self.h = h
        self.N = plan.N
        s = C.c_void_p()
        check(self._lib.lev_get_stream(h, C.byref(s)))
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.ExternalStream(s.value, device=self.device)

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr())

    def tensor(self, n, dtype="float32"):
        import torch

        return torch.zeros(n, dtype=getattr(torch, dtype), device=self.device)

    def upload(self, a, dtype="int32"):
        import torch

        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def step_begin(self, dt, partials):
        self._check(self._lib.lev_part_step_begin(self.h, float(dt), self._p(partials)))

    def step_end(self, dt, partials_all, r_slot):
        self._check(self._lib.lev_part_step_end(self.h, float(dt), self._p(partials_all),
                                                self._p(r_slot)))

    # two steps per pair of launches (see lev_part_pair_begin)
    def pairs_eligible(self) -> bool:
        el = C.c_int32()
        self._check(self._lib.lev_part_pairs(self.h, C.byref(el)))
        return bool(el.value)

    def pair_begin(self, dt, partials):
        self._check(self._lib.lev_part_pair_begin(self.h, float(dt), self._p(partials)))

    def pair_finish(self, dt, partials):
        self._check(self._lib.lev_part_pair_finish(self.h, float(dt), self._p(partials)))

    def pack(self, idx, out):
        self._check(self._lib.lev_part_pack(self.h, self._p(idx), int(idx.numel()),
                                            self._p(out)))

    def unpack(self, idx, inp):
        self._check(self._lib.lev_part_unpack(self.h, self._p(idx), int(idx.numel()),
                                              self._p(inp)))

    def synchronize(self):
        self._check(self._lib.lev_sync(self.h))

    def get_theta(self):
        out = np.empty(self.N, np.float32)
        self._check(self._lib.lev_get_theta(self.h, C.c_void_p(out.ctypes.data)))
        return out

    def get_weights(self):
        from ._lib import load

        E = C.c_int64()
        self._check(load().lev_total_edges(self.h, C.byref(E)))
        out = np.empty(max(E.value, 1), np.float32)
        self._check(self._lib.lev_get_weights(self.h, C.c_void_p(out.ctypes.data)))
        return out[:E.value]

    def get_gain(self):
        g = C.c_float()
        self._check(self._lib.lev_get_gain(self.h, 0, C.byref(g)))
        return g.value

    def set_theta(self, theta_own, theta_halo):
        a = np.ascontiguousarray(theta_own, np.float32)
        b = np.ascontiguousarray(theta_halo, np.float32)
        self._check(self._lib.lev_set_theta(self.h, C.c_void_p(a.ctypes.data)))
        self._check(self._lib.lev_part_fill_halo(self.h, C.c_void_p(b.ctypes.data)
                                                 if b.size else C.c_void_p(0)))

    def close(self):
        if self.h:
            self._lib.lev_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# the halo engine of one rank
# ---------------------------------------------------------------------------
class PartitionedEngine:
    """Rank ``rank``'s part of one network that is stepped by ``world``
    ranks together.  Every rank constructs it with the whole network's
    arrays (``engine_args`` order of the reference constructor) and calls
    the same methods in the same order.

    ``exchange``: :class:`DistExchange` (one process per GPU) or a
    :class:`ThreadExchange` binding.  ``core``: per-rank compute class,
    :class:`CudaPartition` unless a test substitutes its own."""

    def __init__(self, rank, world, N, max_delay, row_ptr, col_idx, delays, weights,
                 theta, theta_hat, omega, *, exchange, params=None,
                 math_mode="reference", plan: PartitionPlan | None = None,
                 core=CudaPartition):
        if isinstance(math_mode, str):
            math_mode = {"reference": 0, "accurate": 1}[math_mode]
        self.plan = plan if plan is not None else PartitionPlan(row_ptr, col_idx, world)
        if self.plan.world != world or self.plan.N != int(N):
            raise ValueError("partition plan does not match world / N")
        pr = self.plan.rank(rank)
        self.rank, self.world, self.pr = rank, world, pr
        theta = np.asarray(theta, np.float32)
        self.core = core(pr, np.asarray(delays)[pr.edge0:pr.edge1],
                         np.asarray(weights)[pr.edge0:pr.edge1],
                         theta[pr.row0:pr.row1], np.asarray(theta_hat)[pr.row0:pr.row1],
                         np.asarray(omega)[pr.row0:pr.row1], theta[pr.halo],
                         max_delay, params=params, math_mode=math_mode)
        self.exchange = exchange
        C_ = pr.tiles_per_rank
        self._part_all = self.core.tensor(world * C_ * 2)
        self._chunk = self._part_all[2 * rank * C_: 2 * (rank + 1) * C_]
        self._send_idx = {p: self.core.upload(v) for p, v in pr.send.items()}
        self._recv_idx = {p: self.core.upload(v) for p, v in pr.recv.items()}
        self._send_buf = {p: self.core.tensor(v.size) for p, v in pr.send.items()}
        self._recv_buf = {p: self.core.tensor(v.size) for p, v in pr.recv.items()}
        self._r_hist = self.core.tensor(256)
        self.steps = 0
        # two steps per pair of launches when every rank's core can take
        # them (no zero delay anywhere: each rank checks its own edges); the
        # ranks agree through one all-gather, so they issue the same
        # collectives in the same order
        ok = hasattr(self.core, "pair_begin") and self.core.pairs_eligible()
        flags = self.core.tensor(world)
        flags[rank:rank + 1].fill_(1.0 if ok else 0.0)
        self.exchange.allgather(flags, flags[rank:rank + 1].clone(), stream=None)
        self._pairs_ok = bool(flags.min().item() > 0.0)
        self._pairs = self._pairs_ok

    @property
    def stream(self):
        return getattr(self.core, "stream", None)

    def _halo(self):
        """theta after the last step -> the peers' halo columns of its slot."""
        core, ex, st = self.core, self.exchange, self.stream
        for p, idx in self._send_idx.items():
            core.pack(idx, self._send_buf[p])
        ex.exchange(self._send_buf, self._recv_buf, stream=st)
        for p, idx in self._recv_idx.items():
            core.unpack(idx, self._recv_buf[p])

    def _one_step(self, dt, r_slot):
        core, ex, st = self.core, self.exchange, self.stream
        # the rank's tiles land at their global positions, inside its chunk
        core.step_begin(dt, self._part_all)
        ex.allgather(self._part_all, self._chunk, stream=st)
        core.step_end(dt, self._part_all, r_slot)
        self._halo()
        self.steps += 1

    def _one_pair(self, dt, r_slots):
        """Steps t, t+1 (lev_part_pair_begin): the halo gets theta(t+1)
        before the finish overwrites it, then theta(t+2)."""
        core, ex, st = self.core, self.exchange, self.stream
        core.pair_begin(dt, self._part_all)
        ex.allgather(self._part_all, self._chunk, stream=st)
        core.step_end(dt, self._part_all, r_slots[0:1])
        self._halo()
        core.pair_finish(dt, self._part_all)
        ex.allgather(self._part_all, self._chunk, stream=st)
        core.step_end(dt, self._part_all, r_slots[1:2])
        self._halo()
        self.steps += 2

    def set_pair_mode(self, enabled: bool) -> None:
        """Two steps per pair of launches (when every rank can), or one step
        per launch.  Every rank must make the same call."""
        self._pairs = bool(enabled) and self._pairs_ok

    def step_n(self, dt, n) -> np.ndarray:
        """``n`` steps; returns r of every step (the same on every rank)."""
        n = int(n)
        if self._r_hist.numel() < n:
            self._r_hist = self.core.tensor(n)
        k = 0
        while k < n:
            if self._pairs and k + 1 < n:
                self._one_pair(dt, self._r_hist[k:k + 2])
                k += 2
            else:
                self._one_step(dt, self._r_hist[k:k + 1])
                k += 1
        self.core.synchronize()
        return self._r_hist[:n].cpu().numpy().copy()

    def step(self, dt) -> float:
        return float(self.step_n(dt, 1)[0])

    # -- state --------------------------------------------------------------
    def get_theta(self) -> np.ndarray:
        """Phases of this rank's own rows."""
        return self.core.get_theta()

    def gather_theta(self) -> np.ndarray:
        """Phases of the whole network (every rank gets them)."""
        import torch

        C_ = self.pr.tiles_per_rank * TILE
        own = self.core.get_theta()
        chunk = torch.zeros(C_, dtype=torch.float32, device=self._part_all.device)
        chunk[:own.size] = torch.from_numpy(own).to(chunk.device)
        out = torch.zeros(self.world * C_, dtype=torch.float32, device=chunk.device)
        self.exchange.allgather(out, chunk, stream=None)
        full = out.cpu().numpy()
        return np.concatenate([full[r * C_: r * C_ + (b1 - b0)]
                               for r, (b0, b1) in enumerate(self.plan.bounds)])

    def get_weights(self) -> np.ndarray:
        """Weights of this rank's own rows' edges (global CSR order)."""
        return self.core.get_weights()

    def get_gain(self) -> float:
        return self.core.get_gain()

    def set_theta(self, theta) -> None:
        """Whole-network phases (every rank passes the same array); every
        ring slot is refilled (leviathan_set_theta, leviathan_kernel.cu:
        445-453), the halo columns included."""
        th = np.asarray(theta, np.float32)
        self.core.set_theta(th[self.pr.row0:self.pr.row1], th[self.pr.halo])

    def close(self):
        self.core.close()
