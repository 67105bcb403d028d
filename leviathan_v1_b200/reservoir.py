"""Differentiable reservoir: the network as a trainable dynamical substrate.

The reference uses the engine as a reservoir by kicking phases through
``set_theta`` and reading cos/sin features back to the host every step
(python/reservoir.py:46-61), with a Ridge readout (:77-87).  Here input and
readout stay on the device and are differentiable end to end:

* a batch of B copies of one network (one ``BatchEngine``), copy b driven by
  its own input sequence x_b(t);
* drive  u_i(t) = W_in[i] * x_b(t) on the input nodes (trainable W_in),
  added to d theta_i / dt -- fused into the step kernel;
* readout y_b(t) = sum_i a_i cos theta_i(t+1) + b_i sin theta_i(t+1) + c --
  reduced inside the step kernel, so no [T, N] array is materialised;
* gradients w.r.t. W_in, omega, the readout (a, b) -- by the adjoint kernels
  (``lev_adj_backward``) through ``torch.autograd``.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .adjoint import Adjoint, _p
from .engine import BatchEngine
from .graphs import Network
from ._lib import check


class _ReservoirRun(torch.autograd.Function):
    @staticmethod
    def forward(ctx, omega, w0, K, win, ra, rb, x, adj, T, dt):
        lib = adj.lib
        B = adj.num_nets
        y = torch.empty((T, B), dtype=torch.float32, device=omega.device)
        win, ra, rb = win.contiguous(), ra.contiguous(), rb.contiguous()
        x = x.contiguous()
        check(lib.lev_adj_set_reservoir(adj._h, _p(win), _p(x), _p(ra), _p(rb), _p(y)))
        r = adj.forward(omega, w0, K, T, dt)
        ctx.adj = adj
        ctx.keep = (win, ra, rb, x)  # the kernels read them again in backward
        return y, r

    @staticmethod
    def backward(ctx, grad_y, grad_r):
        adj = ctx.adj
        lib = adj.lib
        dev = grad_y.device if grad_y is not None else grad_r.device
        n = adj.total_nodes
        g_win = torch.empty(n, dtype=torch.float32, device=dev)
        g_ra = torch.empty(n, dtype=torch.float32, device=dev)
        g_rb = torch.empty(n, dtype=torch.float32, device=dev)
        gy = grad_y.contiguous().float() if grad_y is not None else None
        check(lib.lev_adj_set_reservoir_grads(adj._h, _p(gy), _p(g_win), _p(g_ra), _p(g_rb)))
        g = adj.backward(grad_r)
        check(lib.lev_adj_set_reservoir_grads(adj._h, None, None, None, None))
        return g["omega"], g["w0"], g["K"], g_win, g_ra, g_rb, None, None, None, None


def make_inputs(batch: int, T: int, seed: int = 0, noise: float = 0.05,
                p_lo: float = 20.0, p_hi: float = 200.0) -> np.ndarray:
    """Input sequences x_b(t) = sum of 3 sinusoids (periods uniform in
    [p_lo, p_hi] steps, random phases) + Gaussian noise; [batch, T]."""
    rng = np.random.default_rng([seed, 0x5E9])
    t = np.arange(T, dtype=np.float64)
    out = np.empty((batch, T))
    for b in range(batch):
        P = rng.uniform(p_lo, p_hi, 3)
        phi = rng.uniform(0, 2 * np.pi, 3)
        out[b] = np.sin(2 * np.pi * t[None, :] / P[:, None] + phi[:, None]).sum(0)
        out[b] += rng.normal(0.0, noise, T)
    return out.astype(np.float32)


class DifferentiableReservoir(torch.nn.Module):
    """B copies of ``net`` as a reservoir with trainable input weights,
    natural frequencies and cos/sin readout."""

    def __init__(self, net: Network, batch: int, n_input: int = 256, T: int = 1000,
                 segment: int = 50, seed: int = 0, math_mode: str = "accurate",
                 params: dict | None = None, device: str = "cuda"):
        super().__init__()
        self.net = net
        self.B = int(batch)
        self.N = net.N
        self.T = int(T)
        self.engine = BatchEngine([net.as_dict()] * self.B,
                                  params=[params or {}] * self.B, math_mode=math_mode)
        self.adj = Adjoint(self.engine, segment=segment, max_steps=self.T)
        rng = np.random.default_rng([seed, 0x1AB])
        self.input_nodes = torch.as_tensor(np.sort(rng.choice(self.N, n_input, replace=False)),
                                           device=device)
        self.w_in = torch.nn.Parameter(torch.tensor(rng.normal(0, 1.0, n_input),
                                                    dtype=torch.float32, device=device))
        self.omega = torch.nn.Parameter(torch.tensor(net.omega, device=device))
        self.register_buffer("w0", torch.tensor(net.weights, device=device))
        # small random readout: with an all-zero readout no gradient reaches
        # the dynamics (W_in, omega) until the readout itself has moved
        ro = rng.normal(0.0, 1.0 / math.sqrt(2 * self.N), (2, self.N))
        self.read_a = torch.nn.Parameter(torch.tensor(ro[0], dtype=torch.float32, device=device))
        self.read_b = torch.nn.Parameter(torch.tensor(ro[1], dtype=torch.float32, device=device))
        self.read_c = torch.nn.Parameter(torch.zeros(1, device=device))
        self.K = float((params or {}).get("g", 1.5))

    def forward(self, x: torch.Tensor, dt: float = 0.05):
        """x [B, T] -> predictions y [B, T] and order parameters r [B, T]."""
        B, T, N = self.B, x.shape[1], self.N
        win = torch.zeros(B, N, device=x.device, dtype=torch.float32)
        win = win.index_copy(1, self.input_nodes, self.w_in.expand(B, -1)).reshape(-1)
        omega = self.omega.repeat(B)
        w0 = self.w0.repeat(B)
        K = torch.full((B,), self.K, device=x.device, dtype=torch.float32)
        ra = self.read_a.repeat(B)
        rb = self.read_b.repeat(B)
        xt = x.t().contiguous().float()  # [T, B]
        y, r = _ReservoirRun.apply(omega, w0, K, win, ra, rb, xt, self.adj, int(T), float(dt))
        return y.t() + self.read_c, r.t()

    @staticmethod
    def loss(y: torch.Tensor, x: torch.Tensor, horizon: int = 10):
        """MSE of predicting x(t + horizon) from the readout at t."""
        return torch.mean((y[:, :-horizon] - x[:, horizon:]) ** 2)

    def close(self):
        self.adj.close()
        self.engine.close()
