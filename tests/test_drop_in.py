"""Drop-in checks of the boundary.

* The reference's own pybind11 binding (src/bindings/leviathan_pybind11.cpp,
  unmodified) compiled against this repository's libleviathan_b200.so by
  oracle/Makefile (into oracle/_ref/b200_binding/): it loads, exposes the
  reference's methods, and -- on a GPU -- reproduces the reference engine's
  golden outputs bit for bit.
* ``LeviathanObservatory``: the reference host API on this engine.
"""

import os
import sys

import numpy as np
import pytest

from conftest import REPO, golden_cases, has_gpu, load_golden, network_from_golden

BINDING_DIR = os.path.join(REPO, "oracle", "_ref", "b200_binding")
DT = 0.05


def _binding():
    if not os.path.isdir(BINDING_DIR) or not os.listdir(BINDING_DIR):
        pytest.skip("reference binding not built (make -C oracle)")
    if BINDING_DIR not in sys.path:
        sys.path.insert(0, BINDING_DIR)
    import leviathan_cuda

    assert os.path.dirname(leviathan_cuda.__file__) == BINDING_DIR
    return leviathan_cuda


def test_reference_binding_links_against_this_library():
    mod = _binding()
    E = mod.LeviathanEngine
    for name in ("step", "get_theta", "set_theta", "set_gain", "get_gain",
                 "set_gain_controller", "get_vram_usage", "reset_weights"):
        assert hasattr(E, name), name
    # the binding resolves the reference symbols in libleviathan_b200.so
    with open(f"/proc/{os.getpid()}/maps") as f:
        maps = f.read()
    assert "libleviathan_b200.so" in maps


@pytest.mark.gpu
@pytest.mark.skipif("c0" not in golden_cases(), reason="golden vectors not generated")
def test_reference_binding_on_this_engine_reproduces_reference_golden():
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    mod = _binding()
    z = load_golden("c0")
    net = network_from_golden(z)
    e = mod.LeviathanEngine(*net.engine_args())
    r = np.array([e.step(DT) for _ in range(500)], np.float32)
    np.testing.assert_array_equal(r, z["r"])
    np.testing.assert_array_equal(e.get_theta(), z["theta@500"])
    # the reference's set_theta semantics (size check raises RuntimeError)
    with pytest.raises(RuntimeError):
        e.set_theta(np.zeros(3, np.float32))
    e.set_gain(2.0)
    assert e.get_gain() == np.float32(2.0)
    assert e.get_vram_usage() > 0
    del e


@pytest.mark.gpu
def test_observatory_runs_like_the_reference_host_api():
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200 import LeviathanObservatory

    a = LeviathanObservatory(N=2000, k=10, max_delay=20, seed=1, verbose=False)
    b = LeviathanObservatory(N=2000, k=10, max_delay=20, seed=1, verbose=False)
    ra = a.run_baseline(num_steps=300, log_interval=100).copy()
    rb = np.array([b.step() for _ in range(300)], np.float32)
    np.testing.assert_array_equal(ra, rb)  # step blocks == single steps
    nodes = [3, 7, 7, 1999]  # a repeated node is kicked twice
    rs = a.run_with_stimulus(num_steps=120, stimulus_start=64, stimulus_nodes=nodes,
                             stimulus_strength=2.5)
    # the reference's loop (python/leviathan_h100.py:178-189): one step per
    # call, the kick after step index stimulus_start
    ref = []
    for i in range(120):
        ref.append(b.step())
        if i == 64:
            th = b.get_phase_snapshot()
            for n in nodes:
                th[n] += 2.5
            b.set_phase_snapshot(th % (2 * np.pi))
    np.testing.assert_array_equal(rs, np.array(ref, np.float32))
    np.testing.assert_array_equal(a.get_phase_snapshot(), b.get_phase_snapshot())
    assert rs.shape == (120,) and a.step_count == 420
    st = a.statistics()
    assert st["steps"] == 420 and 0 <= st["min_r"] <= st["max_r"] <= 1
    th = a.get_phase_snapshot()
    assert th.shape == (2000,) and np.all((th >= 0) & (th < 2 * np.pi + 1e-5))
    a.set_phase_snapshot(np.zeros(2000))
    np.testing.assert_array_equal(a.get_phase_snapshot(), np.zeros(2000, np.float32))
    a.set_gain_controller(False)
    a.set_gain(3.0)
    assert a.get_gain() == np.float32(3.0)
    a.step()
    assert a.get_gain() == np.float32(3.0)  # controller off
    assert "TOTAL (Measured)" in a.get_vram_report()
    a.reset_weights()
    a.close()
    b.close()
