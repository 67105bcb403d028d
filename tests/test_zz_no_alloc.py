"""The allocation-free step ``lev_step_noalloc`` (GPU).

Some callers cannot allocate device memory themselves -- their memory is
owned by a planner or a framework allocator, or they run in loops where
cudaMalloc's device-wide synchronisation is not acceptable -- so they keep
every buffer of the network and call a step that allocates nothing.  This
test plays such a caller: it owns the buffers (allocated here with torch, as
the caller's own allocator would), calls the entry point through the C ABI
twice in a row, and compares each result with the engine's own ``lev_step``
on the same network, within the tolerances of the engine parity tests.

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


def test_noalloc_step_matches_engine_step_twice():
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    import torch

    from leviathan_v1_b200 import LeviathanEngine, _lib
    from leviathan_v1_b200.graphs import make_network

    lib = _lib.load()
    net = make_network(20_000, 16, 0.1, 30, seed=21)
    N, md = net.N, net.max_delay
    bsi = md + 2
    eng = LeviathanEngine(*net.engine_args())

    dev = torch.device("cuda", torch.cuda.current_device())
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    row_ptr, col, dl = T(net.row_ptr), T(net.col_idx), T(net.delays)
    w, th, thh = T(net.weights), T(net.theta), T(net.theta_hat)
    om, omh = T(net.omega), T(net.omega.copy())
    ring = th.repeat(bsi)  # every slot := theta
    gain = torch.tensor([1.5], dtype=torch.float32, device=dev)
    r_out = torch.zeros(1, dtype=torch.float32, device=dev)
    P = lambda x: C.c_void_p(x.data_ptr())
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()

    for t in range(2):
        rc = lib.lev_step_noalloc(N, md, t, P(row_ptr), P(col), P(dl), P(w), P(th),
                                  P(thh), P(om), P(omh), P(ring), P(gain), P(r_out),
                                  None, C.c_float(DT), 0, C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.lev_last_error().decode()
        torch.cuda.synchronize()
        r_eng = eng.step(DT)
        assert abs(float(r_out.item()) - r_eng) <= TOL["r"]
        assert circular_distance(th.cpu().numpy(), eng.get_theta()).max() <= TOL["theta"]
        assert np.abs(w.cpu().numpy() - eng.get_weights()).max() <= TOL["w"]
        th_hat, om_hat = eng.get_predictor()
        assert np.abs(thh.cpu().numpy() - th_hat).max() <= TOL["hat"]
        assert np.abs(omh.cpu().numpy() - om_hat).max() <= TOL["hat"]
        assert abs(float(gain.item()) - eng.get_gain()) <= TOL["g"]
        # the caller's ring holds theta(t+1) in slot (t+1) mod (max_delay+2)
        slot = (t + 1) % bsi
        assert circular_distance(ring[slot * N:(slot + 1) * N].cpu().numpy(),
                                 eng.get_theta()).max() <= TOL["theta"]
    eng.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200 import _lib

    lib = _lib.load()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.lev_step_noalloc((1 << 22) + 1, 10, 0, dummy, dummy, dummy, dummy,
                              dummy, dummy, dummy, dummy, dummy, dummy, dummy,
                              None, C.c_float(DT), 0, None)
    assert rc == _lib.LEV_ERR_ARG
    assert "4194304" in lib.lev_last_error().decode()
