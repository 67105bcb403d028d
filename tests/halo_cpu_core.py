"""FP32 NumPy stand-in for one rank's compute in the halo engine.

TEST INFRASTRUCTURE ONLY: ``PartitionedEngine(core=CpuPartitionCore)`` lets
the multi-rank data plane (partition plan, all-gather of tile partials,
halo send/recv, r and the controller from the gathered partials) run as
gloo ranks on a machine without a GPU.  It has the interface of
``leviathan_v1_b200.halo.CudaPartition`` and the equations of the FP64
oracle (oracle/oracle64.py, which follows leviathan_kernel.cu:93-264 and
:431-435), evaluated in float32 with a fixed summation order:

* the coupling sum of a row is accumulated edge by edge in CSR order;
* tile partials are the 32-lane shuffle-down tree of each warp, then the
  same tree over the eight warp sums (leviathan_kernel.cu:198-233);
* r is formed from all tile partials lane-strided then by the same tree
  (:242-263).

So a partitioned run and an unpartitioned run of this core agree bit for bit
exactly when the data plane delivers every delayed phase and every partial
where it belongs.
"""

from __future__ import annotations

import numpy as np
import torch

from oracle64 import DEFAULT_PARAMS

F = np.float32
TWO_PI = F(2.0 * np.pi)
TILE = 256


def _wrap_pm(x):
    return (x - np.floor(x / TWO_PI + F(0.5)) * TWO_PI).astype(F)


def _wrap_02(x):
    return (x - np.floor(x / TWO_PI) * TWO_PI).astype(F)


def _tree32(v):
    """Lane 0 of a 32-lane shuffle-down sum tree over the last axis."""
    for off in (16, 8, 4, 2, 1):
        v = v[..., :off] + v[..., off:2 * off]
    return v[..., 0]


def tile_partials(c, s):
    """(sum cos, sum sin) of every 256-node tile, in the block tree order."""
    n = c.size
    T = -(-n // TILE)
    out = []
    for v in (c, s):
        pad = np.zeros(T * TILE, F)
        pad[:n] = v
        warps = _tree32(pad.reshape(T, 8, 32))                # [T, 8]
        lanes = np.zeros((T, 32), F)
        lanes[:, :8] = warps
        out.append(_tree32(lanes))
    return np.stack(out, axis=1)                              # [T, 2]


def reduce_partials(p):
    """r numerator terms from [T, 2] partials: lane-strided then tree."""
    T = p.shape[0]
    lanes = np.zeros((32, 2), F)
    for k in range(T):
        lanes[k % 32] = lanes[k % 32] + p[k]
    return _tree32(lanes[:, 0]), _tree32(lanes[:, 1])


class CpuPartitionCore:
    def __init__(self, plan, delays, weights, theta, theta_hat, omega, theta_halo,
                 max_delay, params=None, math_mode=0):
        p = dict(DEFAULT_PARAMS)
        p.update(params or {})
        self.p = {k: F(v) for k, v in p.items()}
        self.ctrl = bool(p["gain_controller"])
        self.N, self.nh = plan.N, plan.n_halo
        self.bsi = int(max_delay) + 2
        self.rp = np.asarray(plan.row_ptr, np.int64)
        self.col = np.asarray(plan.col_idx, np.int64)
        self.dl = np.asarray(delays, np.int64)
        self.deg = np.diff(self.rp)
        self.row = np.repeat(np.arange(self.N), self.deg)
        self.w = np.array(weights, F)
        self.theta = np.array(theta, F)
        self.theta_hat = np.array(theta_hat, F)
        self.omega = np.array(omega, F)
        self.omega_hat = self.omega.copy()
        self.ring = np.empty((self.bsi, self.N + self.nh), F)
        self.ring[:, :self.N] = self.theta
        self.ring[:, self.N:] = np.asarray(theta_halo, F)
        self.cur = 0
        self.g = self.p["g"]
        self.tile_off = plan.tile_off
        self.ntiles_global = plan.ntiles_global
        self.N_global = plan.N_global
        self._eps = None

    # buffers of the engine: host tensors
    def tensor(self, n, dtype="float32"):
        return torch.zeros(n, dtype=getattr(torch, dtype))

    def upload(self, a):
        return torch.from_numpy(np.ascontiguousarray(a))

    def step_begin(self, dt, partials):
        p, dt = self.p, F(dt)
        with np.errstate(invalid="ignore", over="ignore"):
            eps = np.sin(_wrap_pm(self.theta - self.theta_hat)).astype(F)
            self.theta_hat = (self.theta_hat + dt * self.omega_hat).astype(F)
            self.omega_hat = (self.omega_hat + p["kappa_w"] * dt * eps).astype(F)
            slot = (self.cur - self.dl) % self.bsi
            d = _wrap_pm(self.ring[slot, self.col] - self.theta[self.row])
            sin_d, cos_d = np.sin(d).astype(F), np.cos(d).astype(F)
            terms = (self.w * sin_d).astype(F)
            S = np.zeros(self.N, F)
            for k in range(int(self.deg.max(initial=0))):
                rows = np.flatnonzero(self.deg > k)
                S[rows] = S[rows] + terms[self.rp[rows] + k]
            ae = np.abs(eps)[self.row]
            w = self.w + dt * (p["eta"] * cos_d * (F(1) - p["gamma"] * ae) - p["lam"] * self.w)
            w = np.where(np.isfinite(w), w, p["w_min"])
            self.w = np.clip(w, p["w_min"], p["w_max"]).astype(F)
            x = _wrap_02(self.theta + dt * (self.omega + self.g * S - p["alpha_eps"] * eps))
            x = np.where(np.isfinite(x), x, F(0)).astype(F)
        self.theta = x
        self.ring[(self.cur + 1) % self.bsi, :self.N] = x
        part = tile_partials(np.cos(x).astype(F), np.sin(x).astype(F))
        view = partials.numpy().reshape(-1, 2)
        view[self.tile_off:self.tile_off + part.shape[0]] = part

    def step_end(self, dt, partials_all, r_slot):
        p, dt = self.p, F(dt)
        allp = partials_all.numpy().reshape(-1, 2)[:self.ntiles_global]
        c, s = reduce_partials(allp)
        r = F(np.sqrt(c * c + s * s) * (F(1) / F(self.N_global)))
        if self.ctrl:
            g = self.g + dt * (p["beta"] * (p["r0"] - r) - p["mu"] * (self.g - p["g_rest"]))
            self.g = F(min(max(g, p["g_min"]), p["g_max"]))
        r_slot.numpy()[0] = r
        self.cur = (self.cur + 1) % self.bsi

    # two steps per pair of launches: the same arithmetic in this stand-in
    # (the second step runs whole in pair_finish, after g(t+1) is known and
    # theta(t+1) went to the peers), so a partitioned pair run checks the
    # order of the data plane: theta(t+1) must be packed before the finish
    # overwrites it
    def pairs_eligible(self):
        return bool(self.dl.size == 0 or self.dl.min() > 0)

    def pair_begin(self, dt, partials):
        self.step_begin(dt, partials)

    def pair_finish(self, dt, partials):
        self.step_begin(dt, partials)

    def pack(self, idx, out):
        out.numpy()[:] = self.theta[idx.numpy()]

    def unpack(self, idx, inp):
        self.ring[self.cur, self.N + idx.numpy()] = inp.numpy()

    def synchronize(self):
        pass

    def get_theta(self):
        return self.theta.copy()

    def get_weights(self):
        return self.w.copy()

    def get_gain(self):
        return float(self.g)

    def set_theta(self, theta_own, theta_halo):
        self.theta = np.array(theta_own, F)
        self.ring[:, :self.N] = self.theta
        self.ring[:, self.N:] = np.asarray(theta_halo, F)

    def close(self):
        pass
