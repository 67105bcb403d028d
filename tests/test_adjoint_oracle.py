"""The FP64 autograd gradient reference against the FP64 oracle (CPU):
forward identical, gradients equal to central finite differences."""

import numpy as np
import torch

from adjoint64 import loss_and_grads, simulate, target_sinusoid
from leviathan_v1_b200.graphs import Network, make_network
from oracle64 import OracleEngine

DT = 0.05


def _loss_oracle(net, omega, w0, K, T, params=None):
    n2 = Network(net.N, net.max_delay, net.row_ptr, net.col_idx, net.delays, w0,
                 net.theta, net.theta_hat, omega)
    p = dict(params or {})
    p["g"] = K
    o = OracleEngine(*n2.engine_args(), params=p)
    return float(np.mean((o.run(DT, T) - target_sinusoid(T)) ** 2))


def test_autograd_forward_equals_oracle():
    net = make_network(120, 6, 0.1, 9, seed=2)
    om = torch.tensor(net.omega.astype(np.float64))
    w0 = torch.tensor(net.weights.astype(np.float64))
    r = simulate(net, om, w0, torch.tensor(1.5, dtype=torch.float64), 40).numpy()
    o = OracleEngine(*net.engine_args())
    assert np.abs(r - o.run(DT, 40)).max() < 1e-12


def test_autograd_gradients_match_finite_differences():
    net = make_network(80, 6, 0.1, 7, seed=5)
    T = 40
    L, g_om, g_w, g_K, _ = loss_and_grads(net, T)
    rng = np.random.default_rng(1)
    om = net.omega.astype(np.float64)
    w0 = net.weights.astype(np.float64)
    h = 1e-6
    v = rng.normal(size=om.size)
    fd = (_loss_oracle(net, om + h * v, w0, 1.5, T) - _loss_oracle(net, om - h * v, w0, 1.5, T)) / (2 * h)
    assert abs(fd - g_om @ v) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
    v = rng.normal(size=w0.size) * 0.01
    fd = (_loss_oracle(net, om, w0 + h * v, 1.5, T) - _loss_oracle(net, om, w0 - h * v, 1.5, T)) / (2 * h)
    assert abs(fd - g_w @ v) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
    fd = (_loss_oracle(net, om, w0, 1.5 + h, T) - _loss_oracle(net, om, w0, 1.5 - h, T)) / (2 * h)
    assert abs(fd - g_K) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
