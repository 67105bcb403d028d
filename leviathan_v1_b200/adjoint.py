"""Differentiation through the engine: adjoint kernels behind
``torch.autograd.Function``.

No counterpart in the reference (it has no training path).  ``simulate``
runs T steps of every network of an engine from the phases and predictor
phases the engine held when the :class:`Adjoint` was created, with
differentiable inputs

* ``omega``  [total nodes]  natural frequencies (also omega_hat(0) = omega,
  as leviathan_init sets it, leviathan_kernel.cu:350),
* ``w0``     [total edges]  initial edge weights, CSR order of the inputs,
* ``K``      [num_nets]     initial global coupling gain g(0),
* ``drive``  [T, total nodes] or None, added to d theta / dt (input drive),

and returns ``r`` [T, num_nets] (order parameter after each step) and, with
``record_theta``, the phases ``theta`` [T, total nodes].  The backward pass
runs the hand-written adjoint kernels (``lev_adj_backward``): it recomputes
the trajectory segment by segment from checkpoints taken every ``segment``
steps, so memory is O(T/segment) checkpoints plus one segment of history.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Adjoint:
    """Adjoint state for one engine (its topology, parameters and current
    phases as initial conditions)."""

    def __init__(self, engine, segment: int = 50, max_steps: int = 2000):
        self.lib = _lib.load()
        self.engine = engine
        self.segment = int(segment)
        self.max_steps = int(max_steps)
        h = C.c_void_p()
        check(self.lib.lev_adj_create(C.byref(h), engine.handle, self.segment,
                                      self.max_steps))
        self._h = h
        self.total_nodes = engine.total_nodes
        self.total_edges = engine.total_edges
        self.num_nets = engine.num_nets
        self._drive = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.lev_adj_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def grid_info(self) -> dict:
        """Whether checkpoint segments run as grid-resident launches (single
        networks whose CTAs fit on the device at once)."""
        el, en, r, m, pr = (C.c_int32() for _ in range(5))
        check(self.lib.lev_adj_grid_info(self._h, C.byref(el), C.byref(en), C.byref(r),
                                         C.byref(m), C.byref(pr)))
        return dict(eligible=bool(el.value), enabled=bool(en.value), rows_per_cta=r.value,
                    eligible_rows=[R for R in (64, 128, 256) if m.value & R],
                    paired=bool(pr.value))

    def set_grid_mode(self, enabled: bool, rows_per_cta: int = 0) -> None:
        check(self.lib.lev_adj_set_grid_mode(self._h, 1 if enabled else 0, int(rows_per_cta)))

    def set_grid_wait(self, limit_ns: int = 2_000_000_000, extra_arrivals: int = 0) -> None:
        """Bound of the grid-barrier waits of the segments (default 2 s);
        ``extra_arrivals`` > 0 makes every wait run out (tests)."""
        check(self.lib.lev_adj_set_grid_wait(self._h, int(limit_ns), int(extra_arrivals)))

    def set_grid_pairing(self, enabled: bool) -> None:
        """Recompute segment k-1 and reverse segment k in one paired launch
        (when eligible), or in launches of their own."""
        check(self.lib.lev_adj_set_grid_pairing(self._h, 1 if enabled else 0))

    @property
    def device_bytes(self) -> int:
        b = C.c_size_t()
        check(self.lib.lev_adj_bytes(self._h, C.byref(b)))
        return b.value

    def _check(self, t, n, name):
        if t is None:
            return None
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
        if t.numel() != n:
            raise ValueError(f"{name} must have {n} elements, got {t.numel()}")
        return t

    def forward(self, omega, w0, K, T: int, dt: float = 0.05, drive=None,
                record_theta: bool = False):
        T = int(T)
        omega = self._check(omega.detach().contiguous(), self.total_nodes, "omega")
        w0 = self._check(w0.detach().contiguous(), self.total_edges, "w0")
        K = self._check(K.detach().reshape(-1).contiguous(), self.num_nets, "K")
        if drive is not None:
            drive = self._check(drive.detach().contiguous(), T * self.total_nodes, "drive")
        dev = omega.device
        r = torch.empty((T, self.num_nets), dtype=torch.float32, device=dev)
        th = (torch.empty((T, self.total_nodes), dtype=torch.float32, device=dev)
              if record_theta else None)
        torch.cuda.current_stream(dev).synchronize()
        check(self.lib.lev_adj_forward(self._h, C.c_float(dt), T, _p(omega), _p(w0),
                                       _p(K), _p(drive), _p(r), _p(th)))
        self._drive = drive  # must stay alive until backward
        self._T = T
        return (r, th) if record_theta else r

    def backward(self, dLdr=None, dLdtheta=None, want_drive: bool = False):
        T = self._T
        dev = torch.device("cuda", torch.cuda.current_device())
        if dLdr is not None:
            dLdr = self._check(dLdr.detach().float().contiguous(), T * self.num_nets, "dLdr")
        if dLdtheta is not None:
            dLdtheta = self._check(dLdtheta.detach().float().contiguous(),
                                   T * self.total_nodes, "dLdtheta")
        g_om = torch.empty(self.total_nodes, dtype=torch.float32, device=dev)
        g_w = torch.empty(self.total_edges, dtype=torch.float32, device=dev)
        g_K = torch.empty(self.num_nets, dtype=torch.float32, device=dev)
        g_u = (torch.empty((T, self.total_nodes), dtype=torch.float32, device=dev)
               if want_drive else None)
        torch.cuda.current_stream(dev).synchronize()
        check(self.lib.lev_adj_backward(self._h, _p(dLdr), _p(dLdtheta), _p(g_om),
                                        _p(g_w), _p(g_K), _p(g_u)))
        return dict(omega=g_om, w0=g_w, K=g_K, drive=g_u)


class _Run(torch.autograd.Function):
    @staticmethod
    def forward(ctx, omega, w0, K, drive, adj, T, dt, record_theta):
        out = adj.forward(omega, w0, K, T, dt, drive, record_theta)
        ctx.adj = adj
        ctx.record_theta = record_theta
        ctx.has_drive = drive is not None
        ctx.K_shape = K.shape
        return out

    @staticmethod
    def backward(ctx, grad_r, grad_theta=None):
        g = ctx.adj.backward(grad_r, grad_theta if ctx.record_theta else None,
                             want_drive=ctx.has_drive)
        drive_grad = g["drive"] if ctx.has_drive else None
        return (g["omega"], g["w0"], g["K"].reshape(ctx.K_shape), drive_grad,
                None, None, None, None)


def simulate(adj: Adjoint, omega, w0, K, T: int, dt: float = 0.05, drive=None,
             record_theta: bool = False):
    """Differentiable T-step run (see the module docstring)."""
    return _Run.apply(omega, w0, K, drive, adj, int(T), float(dt), bool(record_theta))
