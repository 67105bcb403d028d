"""Adjoint kernels (GPU) against the FP64 torch-autograd reference and FP64
finite differences.

Tolerance (stated and asserted): relative error of each gradient,
||g_gpu - g_ref|| / ||g_ref|| <= 1e-3, on the small instance N = 200, k = 8,
100 steps, loss = mean_t (r(t) - (0.5 + 0.2 sin(2 pi t / 400)))^2.
"""

import numpy as np
import pytest
import torch

from adjoint64 import loss_and_grads, simulate as simulate64, target_sinusoid
from conftest import has_gpu
from leviathan_v1_b200 import BatchEngine, LeviathanEngine
from leviathan_v1_b200.adjoint import Adjoint, simulate
from leviathan_v1_b200.graphs import Network, make_network
from oracle64 import OracleEngine

pytestmark = pytest.mark.gpu

DT = 0.05
REL = 1e-3


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not has_gpu():
        pytest.fail("GPU tests need a CUDA device")


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def _params_gpu(net, dev="cuda", K=1.5, nets=1):
    om = torch.tensor(net.omega, dtype=torch.float32, device=dev, requires_grad=True)
    w0 = torch.tensor(net.weights, dtype=torch.float32, device=dev, requires_grad=True)
    K = torch.full((nets,), K, dtype=torch.float32, device=dev, requires_grad=True)
    return om, w0, K


def _gpu_grads(net, T, math_mode="accurate", segment=50, grid=None, paired=None):
    eng = LeviathanEngine(*net.engine_args(), math_mode=math_mode)
    adj = Adjoint(eng, segment=segment, max_steps=T)
    if grid is not None:  # False: per-step launches; R: grid-resident, R rows per CTA
        adj.set_grid_mode(bool(grid), int(grid) if grid else 0)
        assert adj.grid_info()["enabled"] == bool(grid)
    if paired is not None:  # recompute k-1 and reverse k in one launch, or not
        adj.set_grid_pairing(paired)
        assert adj.grid_info()["paired"] == paired
    om, w0, K = _params_gpu(net)
    r = simulate(adj, om, w0, K, T, DT)[:, 0]
    tgt = torch.tensor(target_sinusoid(T), dtype=torch.float32, device="cuda")
    L = torch.mean((r - tgt) ** 2)
    L.backward()
    out = (float(L.detach()), om.grad.cpu().numpy(), w0.grad.cpu().numpy(), float(K.grad[0]),
           r.detach().cpu().numpy())
    adj.close()
    eng.close()
    return out


def test_adjoint_forward_equals_engine():
    net = make_network(3000, 12, 0.1, 25, seed=4)
    eng = LeviathanEngine(*net.engine_args())
    adj = Adjoint(eng, segment=16, max_steps=80)
    om, w0, K = _params_gpu(net)
    r_adj = adj.forward(om, w0, K, 80, DT).cpu().numpy()[:, 0]
    r_eng = eng.step_n(DT, 80)
    np.testing.assert_array_equal(r_adj, r_eng)
    adj.close()
    eng.close()


@pytest.mark.parametrize("math_mode", ["accurate", "reference"])
def test_gradients_match_fp64_autograd(math_mode):
    net = make_network(200, 8, 0.1, 20, seed=3)
    L64, g_om64, g_w64, g_K64, r64 = loss_and_grads(net, 100)
    L, g_om, g_w, g_K, r = _gpu_grads(net, 100, math_mode)
    assert np.abs(r - r64).max() < 1e-4
    assert abs(L - L64) <= 1e-4 * abs(L64)
    e_om, e_w, e_K = _rel(g_om, g_om64), _rel(g_w, g_w64), _rel(g_K, g_K64)
    assert e_om <= REL and e_w <= REL and e_K <= REL, (e_om, e_w, e_K)


def test_gradients_match_fp64_finite_differences():
    net = make_network(200, 8, 0.1, 20, seed=11)
    T = 100
    _, g_om, g_w, g_K, _ = _gpu_grads(net, T)

    def L(omega, w0, K):
        n2 = Network(net.N, net.max_delay, net.row_ptr, net.col_idx, net.delays, w0,
                     net.theta, net.theta_hat, omega)
        o = OracleEngine(*n2.engine_args(), params=dict(g=K))
        return float(np.mean((o.run(DT, T) - target_sinusoid(T)) ** 2))

    rng = np.random.default_rng(0)
    om = net.omega.astype(np.float64)
    w0 = net.weights.astype(np.float64)
    h = 1e-6
    v = rng.normal(size=om.size)
    fd = (L(om + h * v, w0, 1.5) - L(om - h * v, w0, 1.5)) / (2 * h)
    assert abs(g_om @ v - fd) <= REL * abs(fd)
    v = rng.normal(size=w0.size)
    fd = (L(om, w0 + h * v, 1.5) - L(om, w0 - h * v, 1.5)) / (2 * h)
    assert abs(g_w @ v - fd) <= REL * abs(fd)
    fd = (L(om, w0, 1.5 + h) - L(om, w0, 1.5 - h)) / (2 * h)
    assert abs(g_K - fd) <= REL * abs(fd)


def test_segment_length_does_not_change_gradients():
    net = make_network(500, 10, 0.1, 30, seed=7)
    a = _gpu_grads(net, 120, segment=7)
    b = _gpu_grads(net, 120, segment=50)
    np.testing.assert_array_equal(a[4], b[4])  # identical forward
    for x, y in zip(a[1:4], b[1:4]):
        assert _rel(x, y) < 1e-5  # adjoint-ring atomics: summation order only


@pytest.mark.parametrize("N,k,md,math_mode", [(10_000, 20, 50, "reference"),
                                             (2000, 12, 0, "accurate"),
                                             (3000, 32, 64, "accurate")])
def test_grid_segments_equal_per_step_launches(N, k, md, math_mode):
    """Grid-resident segments (one cooperative launch per checkpoint segment
    forward and backward, the backward recompute paired with the reverse of
    the segment after it, or not) against per-step launches: the forward
    bitwise, the gradients to summation order (adjoint-ring atomics, row and
    CTA sums), for every eligible rows-per-CTA choice; a zero-delay network
    included."""
    net = make_network(N, k, 0.1, md, seed=N + k, delay_lo=min(1, md))
    T = 120
    ref = _gpu_grads(net, T, math_mode, segment=50, grid=False)
    eng = LeviathanEngine(*net.engine_args(), math_mode=math_mode)
    adj = Adjoint(eng, segment=50, max_steps=T)
    info = adj.grid_info()
    adj.close()
    eng.close()
    assert info["eligible"] and info["eligible_rows"] and info["paired"], info
    runs = [(R, True) for R in info["eligible_rows"]] + [(info["eligible_rows"][0], False)]
    for R, paired in runs:
        got = _gpu_grads(net, T, math_mode, segment=50, grid=R, paired=paired)
        np.testing.assert_array_equal(got[4], ref[4], err_msg=f"R={R}")
        assert got[0] == ref[0]
        for x, y in zip(got[1:4], ref[1:4]):
            assert _rel(x, y) < 1e-5, (R, paired, _rel(x, y))


def test_drive_and_phase_output_gradients():
    net = make_network(200, 8, 0.1, 20, seed=13)
    T = 60
    rng = np.random.default_rng(2)
    drive = rng.normal(0, 0.5, (T, net.N))
    wsel = rng.normal(size=net.N)
    # FP64 reference: loss on the phases (readout) and on r
    om64 = torch.tensor(net.omega.astype(np.float64), requires_grad=True)
    w64 = torch.tensor(net.weights.astype(np.float64), requires_grad=True)
    K64 = torch.tensor(1.5, dtype=torch.float64, requires_grad=True)
    d64 = torch.tensor(drive, requires_grad=True)
    r, th = simulate64(net, om64, w64, K64, T, DT, drive=d64, record_theta=True)
    L64 = (torch.cos(th) @ torch.tensor(wsel)).pow(2).mean() + r.mean()
    L64.backward()
    # GPU
    eng = LeviathanEngine(*net.engine_args(), math_mode="accurate")
    adj = Adjoint(eng, segment=20, max_steps=T)
    om, w0, K = _params_gpu(net)
    dg = torch.tensor(drive, dtype=torch.float32, device="cuda", requires_grad=True)
    rg, thg = simulate(adj, om, w0, K, T, DT, drive=dg, record_theta=True)
    ws = torch.tensor(wsel, dtype=torch.float32, device="cuda")
    L = (torch.cos(thg) @ ws).pow(2).mean() + rg[:, 0].mean()
    L.backward()
    assert _rel(dg.grad.cpu().numpy(), d64.grad.numpy()) <= REL
    assert _rel(om.grad.cpu().numpy(), om64.grad.numpy()) <= REL
    assert _rel(w0.grad.cpu().numpy(), w64.grad.numpy()) <= REL
    assert _rel(float(K.grad[0]), float(K64.grad)) <= REL
    adj.close()
    eng.close()


def test_batched_adjoint_equals_separate():
    nets = [make_network(300, 8, 0.1, 15, seed=s) for s in (1, 2)]
    be = BatchEngine([n.as_dict() for n in nets], math_mode="accurate")
    adj = Adjoint(be, segment=25, max_steps=60)
    om = torch.tensor(np.concatenate([n.omega for n in nets]), device="cuda", requires_grad=True)
    w0 = torch.tensor(np.concatenate([n.weights for n in nets]), device="cuda", requires_grad=True)
    K = torch.tensor([1.5, 2.0], device="cuda", requires_grad=True)
    r = simulate(adj, om, w0, K, 60, DT)
    (r ** 2).sum().backward()
    for i, n in enumerate(nets):
        e = LeviathanEngine(*n.engine_args(), math_mode="accurate")
        a = Adjoint(e, segment=25, max_steps=60)
        o2, w2, K2 = _params_gpu(n, K=[1.5, 2.0][i])
        r2 = simulate(a, o2, w2, K2, 60, DT)
        np.testing.assert_array_equal(r2[:, 0].detach().cpu().numpy(),
                                      r[:, i].detach().cpu().numpy())
        (r2 ** 2).sum().backward()
        sl = slice(sum(m.N for m in nets[:i]), sum(m.N for m in nets[:i + 1]))
        assert _rel(om.grad[sl].cpu().numpy(), o2.grad.cpu().numpy()) < 1e-5
        assert abs(float(K.grad[i]) - float(K2.grad[0])) <= 1e-5 * abs(float(K2.grad[0])) + 1e-9
        a.close()
        e.close()
    adj.close()
    be.close()
