"""Differentiable reservoir (fused input drive and cos/sin readout in the
step and adjoint kernels) against an FP64 torch-autograd reference (GPU).

Tolerance (stated and asserted): relative error <= 1e-3 of the gradients
w.r.t. the input weights, omega and the readout weights, on a 200-node
network, batch 3, 60 steps.
"""

import numpy as np
import pytest
import torch

from adjoint64 import simulate as simulate64
from conftest import has_gpu
from leviathan_v1_b200.graphs import make_network
from leviathan_v1_b200.reservoir import DifferentiableReservoir, make_inputs

pytestmark = pytest.mark.gpu

DT = 0.05
REL = 1e-3


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def test_reservoir_gradients_match_fp64_autograd():
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    net = make_network(200, 8, 0.1, 20, seed=17)
    B, T, H = 3, 60, 10
    model = DifferentiableReservoir(net, B, n_input=16, T=T, segment=20, seed=1)
    rng = np.random.default_rng(4)
    with torch.no_grad():
        model.read_a.copy_(torch.tensor(rng.normal(0, 0.05, net.N), dtype=torch.float32))
        model.read_b.copy_(torch.tensor(rng.normal(0, 0.05, net.N), dtype=torch.float32))
        model.read_c.fill_(0.1)
    x = make_inputs(B, T, seed=3)
    xt = torch.tensor(x, device="cuda")
    y, r = model(xt, DT)
    L = model.loss(y, xt, H) + 0.1 * r.mean()
    L.backward()

    # FP64 reference: batch element b driven by w_in * x_b(t) on the input nodes
    inp = model.input_nodes.cpu().numpy()
    w_in = torch.tensor(model.w_in.detach().cpu().numpy().astype(np.float64), requires_grad=True)
    om = torch.tensor(net.omega.astype(np.float64), requires_grad=True)
    a = torch.tensor(model.read_a.detach().cpu().numpy().astype(np.float64), requires_grad=True)
    b_ = torch.tensor(model.read_b.detach().cpu().numpy().astype(np.float64), requires_grad=True)
    c = torch.tensor(0.1, dtype=torch.float64, requires_grad=True)
    w0 = torch.tensor(net.weights.astype(np.float64))
    x64 = torch.tensor(x.astype(np.float64))
    ys, rs = [], []
    for bi in range(B):
        drive = torch.zeros(T, net.N, dtype=torch.float64)
        drive = drive.index_copy(1, torch.as_tensor(inp), x64[bi][:, None] * w_in[None, :])
        rb, th = simulate64(net, om, w0, torch.tensor(1.5, dtype=torch.float64), T, DT,
                            drive=drive, record_theta=True)
        ys.append(torch.cos(th) @ a + torch.sin(th) @ b_ + c)
        rs.append(rb)
    Y = torch.stack(ys)
    R = torch.stack(rs)
    L64 = torch.mean((Y[:, :-H] - x64[:, H:]) ** 2) + 0.1 * R.mean()
    L64.backward()

    assert np.abs(y.detach().cpu().numpy() - Y.detach().numpy()).max() < 1e-3
    assert abs(float(L.detach()) - float(L64.detach())) <= 1e-4 * abs(float(L64.detach()))
    errs = dict(w_in=_rel(model.w_in.grad.cpu(), w_in.grad),
                omega=_rel(model.omega.grad.cpu(), om.grad),
                read_a=_rel(model.read_a.grad.cpu(), a.grad),
                read_b=_rel(model.read_b.grad.cpu(), b_.grad),
                read_c=_rel(model.read_c.grad.cpu(), c.grad))
    assert all(v <= REL for v in errs.values()), errs
    model.close()
