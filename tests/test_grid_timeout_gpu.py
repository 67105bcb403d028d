"""The bounded grid-barrier wait of the grid-resident kernels (GPU).

A wait that runs out must end the launch with an error the host reads, not
a hang or a fault.  These tests make every wait run out on purpose: with
``extra_arrivals`` the barrier expects one arrival more than the grid makes,
and the wait limit is 20 microseconds, so each CTA gives up at its first
wait, sets the error flag in mapped host memory and returns.  Nothing here
faults or hangs the GPU; the longest wait is 20 us per CTA.

Checked: the step block returns LEV_ERR_CUDA; the engine stops using the
grid path; the state is that from before the block (the timed-out launch
wrote nothing back), so the next blocks equal a fresh engine on per-step
launches bit for bit.  The same for the adjoint's grid-resident segments.
"""

import numpy as np
import pytest
import torch

from conftest import has_gpu
from leviathan_v1_b200 import LeviathanEngine, _lib
from leviathan_v1_b200.adjoint import Adjoint
from leviathan_v1_b200.graphs import make_network

pytestmark = pytest.mark.gpu

DT = 0.05
LIMIT_NS = 20_000


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not has_gpu():
        pytest.fail("GPU tests need a CUDA device")


def _state(e):
    th_hat, om_hat = e.get_predictor()
    ring, bi = e.get_ring(0)
    return dict(theta=e.get_theta(), w=e.get_weights(), thh=th_hat, omh=om_hat,
                ring=ring, bi=np.array(bi), g=np.array(e.get_gain()))


@pytest.mark.parametrize("md", [50, 0])  # early waits (no zero delay) and late ones
def test_grid_wait_timeout_is_reported_and_state_kept(md):
    net = make_network(10_000, 20, 0.1, md, seed=77, delay_lo=min(1, md))
    ref = LeviathanEngine(*net.engine_args())
    ref.set_cluster_mode(False)
    ref.set_grid_mode(False)
    r_ref = np.concatenate([ref.step_n(DT, 7), ref.step_n(DT, 40)])

    e = LeviathanEngine(*net.engine_args())
    e.set_cluster_mode(False)
    e.set_grid_mode(True)
    assert e.grid_info()["enabled"]
    r0 = e.step_n(DT, 7)  # grid path, normal waits
    np.testing.assert_array_equal(r0, r_ref[:7])
    before = _state(e)
    e.set_grid_wait(LIMIT_NS, extra_arrivals=1)
    with pytest.raises(_lib.LevError) as exc:
        e.step_n(DT, 40)
    assert exc.value.code == _lib.LEV_ERR_CUDA
    assert "timed out" in str(exc.value)
    assert not e.grid_info()["enabled"]  # the engine stopped using the path
    after = _state(e)
    for k in ("theta", "w", "thh", "omh", "bi", "g"):
        np.testing.assert_array_equal(after[k], before[k], err_msg=k)
    e.set_grid_wait()  # default bound again
    r1 = e.step_n(DT, 40)  # per-step launches from the kept state
    np.testing.assert_array_equal(r1, r_ref[7:])
    want, got = _state(ref), _state(e)
    for k in ("theta", "w", "thh", "omh", "ring", "bi", "g"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    e.close()
    ref.close()


def test_grid_wait_arguments_are_checked():
    net = make_network(2000, 8, 0.1, 10, seed=1)
    e = LeviathanEngine(*net.engine_args())
    with pytest.raises(ValueError):
        e.set_grid_wait(10)  # below 1 us
    with pytest.raises(ValueError):
        e.set_grid_wait(LIMIT_NS, extra_arrivals=5000)
    e.close()


def _adj_run(net, T, grid, wait=None):
    eng = LeviathanEngine(*net.engine_args(), math_mode="accurate")
    adj = Adjoint(eng, segment=25, max_steps=T)
    adj.set_grid_mode(grid)
    om = torch.tensor(net.omega, device="cuda", requires_grad=False)
    w0 = torch.tensor(net.weights, device="cuda")
    K = torch.full((1,), 1.5, device="cuda")
    err = None
    if wait is not None:
        adj.set_grid_wait(*wait)
        try:
            adj.forward(om, w0, K, T, DT)
        except _lib.LevError as exc:
            err = exc
        adj.set_grid_wait()
    r = adj.forward(om, w0, K, T, DT).cpu().numpy()
    dLdr = torch.ones(T, 1, device="cuda") / T
    grads = adj.backward(dLdr)
    info = adj.grid_info()
    out = (r, [grads[k].cpu().numpy() for k in ("omega", "w0", "K")], info, err)
    adj.close()
    eng.close()
    return out


def test_adjoint_grid_wait_timeout_is_reported():
    net = make_network(10_000, 20, 0.1, 50, seed=78)
    T = 100
    r_ref, g_ref, _, _ = _adj_run(net, T, grid=False)
    r, g, info, err = _adj_run(net, T, grid=True, wait=(LIMIT_NS, 1))
    assert err is not None and err.code == _lib.LEV_ERR_CUDA
    assert "timed out" in str(err)
    assert not info["enabled"]  # the adjoint stopped using grid segments
    np.testing.assert_array_equal(r, r_ref)  # per-step launches, same trajectory
    # the per-step reverse kernel scatters with atomics, so two runs agree to
    # summation order only
    for a, b in zip(g, g_ref):
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b)
