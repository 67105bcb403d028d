"""FP64 torch-autograd restatement of the engine step, for checking the
adjoint kernels.

TEST INFRASTRUCTURE ONLY (imported by tests/).  It runs the same equations as
``oracle/oracle64.py`` (which follows leviathan_kernel.cu:93-264 and the host
controller :431-435) with torch float64 tensors so that autograd gives the
reference gradients.  Non-smooth points follow the conventions the adjoint
kernels use: the phase wraps (floor) have derivative 1, a clamped weight or
gain passes no gradient, |eps| has derivative sign(eps); the NaN guards are
identity (inputs are finite).  An optional additive drive u[t, i] enters
d theta_i / dt (the reservoir input), and the loss may also read the phases.

Initial conditions as in leviathan_init (:270-389): omega_hat starts equal
to omega (so gradients w.r.t. omega also flow through omega_hat), every ring
slot starts equal to theta(0), the gain starts at K.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from oracle64 import DEFAULT_PARAMS

TWO_PI = 2.0 * math.pi


def _wrap_pm(x):
    return x - torch.floor(x / TWO_PI + 0.5) * TWO_PI


def _wrap_02(x):
    return x - torch.floor(x / TWO_PI) * TWO_PI


def simulate(net, omega, w0, K, T, dt=0.05, params=None, drive=None,
             record_theta=False):
    """Run T steps from (net.theta, net.theta_hat) with parameters
    (omega [N], w0 [E], K scalar) as float64 tensors.  Returns r[T] (r after
    each step) and, if ``record_theta``, the phases theta(1..T) [T, N]."""
    p = dict(DEFAULT_PARAMS)
    if params:
        p.update(params)
    f64 = torch.float64
    N = net.N
    rp = np.asarray(net.row_ptr, np.int64)
    row = torch.as_tensor(np.repeat(np.arange(N), np.diff(rp)), dtype=torch.long)
    col = torch.as_tensor(np.asarray(net.col_idx, np.int64))
    d = torch.as_tensor(np.asarray(net.delays, np.int64))
    bs = int(net.max_delay) + 1
    theta = torch.as_tensor(np.asarray(net.theta, np.float64))
    theta_hat = torch.as_tensor(np.asarray(net.theta_hat, np.float64))
    omega_hat = omega
    w = w0
    g = K
    hist = [theta]
    rs, ths = [], []
    for t in range(T):
        diff = _wrap_pm(theta - theta_hat)
        eps = torch.sin(diff)
        theta_hat = theta_hat + dt * omega_hat
        omega_hat = omega_hat + p["kappa_w"] * dt * eps
        # ring window: slot m holds theta(t - m), theta(0) before time 0
        H = torch.stack([hist[max(t - m, 0)] for m in range(bs)])
        delayed = H[d, col]
        delta = _wrap_pm(delayed - theta[row])
        S = torch.zeros(N, dtype=f64).index_add(0, row, w * torch.sin(delta))
        my_eps = torch.abs(eps)[row]
        w_pre = w + dt * (p["eta"] * torch.cos(delta) * (1.0 - p["gamma"] * my_eps)
                          - p["lam"] * w)
        w = torch.clamp(w_pre, p["w_min"], p["w_max"])
        rate = omega + g * S - p["alpha_eps"] * eps
        if drive is not None:
            rate = rate + drive[t]
        theta = _wrap_02(theta + dt * rate)
        hist.append(theta)
        if len(hist) > bs + 1:
            hist[len(hist) - bs - 2] = None  # free
        C = torch.cos(theta).mean()
        Sn = torch.sin(theta).mean()
        r = torch.sqrt(C * C + Sn * Sn)
        rs.append(r)
        if record_theta:
            ths.append(theta)
        if p["gain_controller"]:
            g = torch.clamp(g + dt * (p["beta"] * (p["r0"] - r) - p["mu"] * (g - p["g_rest"])),
                            p["g_min"], p["g_max"])
    r = torch.stack(rs)
    if record_theta:
        return r, torch.stack(ths)
    return r


def target_sinusoid(T, period=400.0):
    """r*(t) = 0.5 + 0.2 sin(2 pi t / period) for t = 1..T."""
    t = np.arange(1, T + 1, dtype=np.float64)
    return 0.5 + 0.2 * np.sin(2 * np.pi * t / period)


def loss_and_grads(net, T, dt=0.05, params=None, K=1.5, target=None):
    """MSE(r, target) and its FP64 gradients w.r.t. omega, w0 and K."""
    omega = torch.tensor(np.asarray(net.omega, np.float64), requires_grad=True)
    w0 = torch.tensor(np.asarray(net.weights, np.float64), requires_grad=True)
    Kt = torch.tensor(float(K), dtype=torch.float64, requires_grad=True)
    r = simulate(net, omega, w0, Kt, T, dt, params)
    tgt = torch.as_tensor(target_sinusoid(T) if target is None else target)
    L = torch.mean((r - tgt) ** 2)
    L.backward()
    return (float(L.detach()), omega.grad.numpy().copy(), w0.grad.numpy().copy(),
            float(Kt.grad), r.detach().numpy())
