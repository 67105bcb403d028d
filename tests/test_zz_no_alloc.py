"""The allocation-free step ``lev_step_noalloc`` (GPU).

Some callers cannot allocate device memory themselves -- their memory is
owned by a planner or a framework allocator, or they run in loops where
cudaMalloc's device-wide synchronisation is not acceptable -- so they keep
every buffer of the network and call a step that allocates nothing.  These
tests play such a caller: they own the buffers (allocated here with torch, as
the caller's own allocator would), call the entry point through the C ABI
many times in a row, and compare each step with the engine's own ``lev_step``
on the same network, within the tolerances of the engine parity tests.

The runs are longer than the delay ring (40 steps against max_delay + 2 = 32
slots), so every ring slot is rewritten and the wrap of the slot index is
exercised, and the whole caller ring is compared with the engine's ring
after every step.

This file is named to be collected last.
"""

import ctypes as C

import numpy as np
import pytest

from conftest import has_gpu
from oracle64 import circular_distance

pytestmark = pytest.mark.gpu

DT = 0.05
TOL = dict(r=1e-5, theta=1e-4, w=1e-5, hat=1e-4, g=1e-5)
STEPS = 40


class CallerBuffers:
    """Device buffers owned by the caller, in the layout lev_step_noalloc
    takes (slot-major ring of max_delay + 2 slots, every slot = theta)."""

    def __init__(self, net, g0):
        import torch

        self.torch = torch
        dev = torch.device("cuda", torch.cuda.current_device())
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.N, self.md = net.N, net.max_delay
        self.row_ptr, self.col, self.dl = T(net.row_ptr), T(net.col_idx), T(net.delays)
        self.w, self.th, self.thh = T(net.weights), T(net.theta), T(net.theta_hat)
        self.om, self.omh = T(net.omega), T(net.omega.copy())
        self.ring = self.th.repeat(self.md + 2)
        self.gain = torch.tensor([g0], dtype=torch.float32, device=dev)
        self.r_out = torch.zeros(1, dtype=torch.float32, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def step(self, lib, t, params, math_mode):
        P = lambda x: C.c_void_p(x.data_ptr())
        rc = lib.lev_step_noalloc(self.N, self.md, t, P(self.row_ptr), P(self.col), P(self.dl),
                                  P(self.w), P(self.th), P(self.thh), P(self.om), P(self.omh),
                                  P(self.ring), P(self.gain), P(self.r_out),
                                  None if params is None else C.byref(params), C.c_float(DT),
                                  math_mode, C.c_void_p(self.stream.cuda_stream))
        assert rc == 0, lib.lev_last_error().decode()
        self.torch.cuda.synchronize()

    def ring_reference_layout(self, t_next):
        """The caller's ring as [N][max_delay+1] in the reference's slot
        order (theta(t') at slot t' mod (max_delay+1)), for theta(t_next)
        and the max_delay phases before it."""
        bsi, bs = self.md + 2, self.md + 1
        ring = self.ring.cpu().numpy().reshape(bsi, self.N)
        out = np.empty((self.N, bs), np.float32)
        for d in range(bs):
            out[:, (t_next - d) % bs] = ring[(t_next - d) % bsi]
        return out


def _compare(buf, eng, r_eng, t):
    r = float(buf.r_out.item())
    assert abs(r - r_eng) <= TOL["r"], (t, r, r_eng)
    th = eng.get_theta()
    assert circular_distance(buf.th.cpu().numpy(), th).max() <= TOL["theta"], t
    assert np.abs(buf.w.cpu().numpy() - eng.get_weights()).max() <= TOL["w"], t
    th_hat, om_hat = eng.get_predictor()
    assert np.abs(buf.thh.cpu().numpy() - th_hat).max() <= TOL["hat"], t
    assert np.abs(buf.omh.cpu().numpy() - om_hat).max() <= TOL["hat"], t
    assert abs(float(buf.gain.item()) - eng.get_gain()) <= TOL["g"], t
    ring_eng, bi = eng.get_ring(0)
    assert bi == (t + 1) % (buf.md + 1)
    ring_eng = np.asarray(ring_eng).reshape(buf.N, buf.md + 1)
    assert circular_distance(buf.ring_reference_layout(t + 1), ring_eng).max() <= TOL["theta"], t


def _run_against_engine(net, params, math_mode):
    from leviathan_v1_b200 import LeviathanEngine, _lib

    lib = _lib.load()
    eng = LeviathanEngine(*net.engine_args(), params=params,
                          math_mode="accurate" if math_mode else "reference")
    cparams = None if params is None else _lib.make_params(**params)
    buf = CallerBuffers(net, eng.get_gain())
    for t in range(STEPS):
        buf.step(lib, t, cparams, math_mode)
        r_eng = eng.step(DT)
        _compare(buf, eng, r_eng, t)
    eng.close()


def test_noalloc_steps_match_engine_steps_reference_math():
    """Default parameters, reference math, 40 calls in a row."""
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200.graphs import make_network

    _run_against_engine(make_network(20_000, 16, 0.1, 30, seed=21), None, 0)


def test_noalloc_steps_match_engine_steps_accurate_math_custom_params():
    """Accurate math and non-default parameters with the gain controller on
    (the controller moves g every step)."""
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200.graphs import make_network

    params = dict(eta=0.02, lam=0.002, gamma=0.1, alpha_eps=0.2, kappa_w=0.02,
                  w_max=1.5, g=2.0, r0=0.6, beta=0.05, mu=0.02, g_rest=1.2,
                  gain_controller=1)
    _run_against_engine(make_network(3000, 20, 0.1, 30, seed=5), params, 1)


def test_noalloc_skips_out_of_range_edges():
    """An edge whose column or delay is out of range adds nothing and keeps
    its weight: the step equals the engine's step on the network without
    those edges."""
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200 import LeviathanEngine, _lib
    from leviathan_v1_b200.graphs import Network, make_network

    lib = _lib.load()
    good = make_network(2000, 10, 0.1, 30, seed=8)
    N, md = good.N, good.max_delay
    # insert two bad edges into row 5 and one into row 1999
    rows = np.repeat(np.arange(N), np.diff(good.row_ptr))
    bad_rows = np.array([5, 5, 1999])
    bad_col = np.array([N + 7, 3, 2 ** 30], np.int32)
    bad_dl = np.array([1, md + 3, 2], np.uint8)
    bad_w = np.array([0.5, 0.25, 0.75], np.float32)
    all_rows = np.concatenate([rows, bad_rows])
    order = np.argsort(all_rows, kind="stable")  # bad edges last in their rows
    is_bad = order >= good.E
    col = np.concatenate([good.col_idx, bad_col])[order]
    dl = np.concatenate([good.delays, bad_dl])[order]
    w = np.concatenate([good.weights, bad_w])[order]
    row_ptr = np.zeros(N + 1, np.int32)
    row_ptr[1:] = np.cumsum(np.bincount(all_rows, minlength=N))
    bad = Network(N, md, row_ptr, col, dl, w, good.theta, good.theta_hat, good.omega)

    eng = LeviathanEngine(*good.engine_args())
    buf = CallerBuffers(bad, eng.get_gain())
    for t in range(STEPS):
        buf.step(lib, t, None, 0)
        r_eng = eng.step(DT)
        assert abs(float(buf.r_out.item()) - r_eng) <= TOL["r"], t
        assert circular_distance(buf.th.cpu().numpy(), eng.get_theta()).max() <= TOL["theta"]
        wb = buf.w.cpu().numpy()
        np.testing.assert_array_equal(wb[is_bad], w[is_bad])  # untouched
        assert np.abs(wb[~is_bad] - eng.get_weights()).max() <= TOL["w"], t
    eng.close()


def test_noalloc_rejects_sizes_beyond_its_scratch_and_null_pointers():
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200 import _lib

    lib = _lib.load()
    dummy = C.c_void_p(16)  # never dereferenced: the checks come first
    rc = lib.lev_step_noalloc((1 << 22) + 1, 10, 0, dummy, dummy, dummy, dummy,
                              dummy, dummy, dummy, dummy, dummy, dummy, dummy,
                              None, C.c_float(DT), 0, None)
    assert rc == _lib.LEV_ERR_ARG
    assert "4194304" in lib.lev_last_error().decode()
    for k in range(11):  # each device pointer NULL in turn
        ptrs = [dummy] * 11
        ptrs[k] = None
        rc = lib.lev_step_noalloc(100, 10, 0, *ptrs, None, C.c_float(DT), 0, None)
        assert rc == _lib.LEV_ERR_ARG, k
        assert "null" in lib.lev_last_error().decode()
