"""Hub-phase transition counts (the integrated-information front-end of the
reference, src/cuda/leviathan_phi_kernel.cu:60-92).  Integer work:
counts, totals, last state and observation count must match the CPU
restatement (oracle/hubs64.py) exactly."""

import numpy as np
import pytest

from conftest import has_gpu
from hubs64 import HubCounter, hub_state

DT = 0.05


# ---------------------------------------------------------------------------
# oracle (CPU)
# ---------------------------------------------------------------------------
def test_binarisation_thresholds():
    pi_f = np.float32(3.1415926)
    above = np.nextafter(pi_f, np.float32(4))
    assert hub_state([pi_f], [0]) == 0          # not above the constant
    assert hub_state([above], [0]) == 1
    assert hub_state([np.float32(np.pi)], [0]) == 1
    assert hub_state([np.float32(-1.0)], [0]) == 1   # -1 + 2pi > pi
    assert hub_state([np.float32(7.0)], [0]) == 0    # 7 - 2pi < pi
    assert hub_state([np.float32("nan")], [0]) == 0  # NaN compares false
    # bit order: hub i is bit i
    assert hub_state([0.0, 4.0, 0.0, 4.0], [1, 3, 0]) == 0b011


def test_engine_phase_range_against_python_driver():
    """On phases in [0, 2pi) the kernel's float32 test and the Python
    driver's ``hub_phases > np.pi`` on a float32 array
    (leviathan_iit_integration.py:88; NumPy >= 2 compares in float32, i.e.
    against float32(pi) = 3.14159274) differ at one phase only: float32(pi)
    itself, which the kernel counts as above 3.1415926f.  The kernel's rule
    is the one implemented."""
    pi32 = np.float32(np.pi)
    x = np.concatenate([np.linspace(0, 2 * np.pi, 100_001, dtype=np.float32)[:-1],
                        np.array([np.nextafter(pi32, np.float32(0)), pi32,
                                  np.nextafter(pi32, np.float32(4))], np.float32)])
    kernel = np.array([hub_state([v], [0]) for v in x.tolist()])
    driver = (x > np.pi).astype(int)
    assert np.array_equal(np.unique(x[kernel != driver]), np.array([pi32], np.float32))


def test_counter_transitions():
    c = HubCounter([0, 1])
    for th in ([0, 0], [4, 0], [4, 4], [0, 0], [0, 0]):
        c.observe(np.array(th, np.float32))
    assert c.observed == 5 and c.prev == 0
    assert c.totals.sum() == 4
    assert c.counts[0, 1] == 1 and c.counts[1, 3] == 1 and c.counts[3, 0] == 1
    assert c.counts[0, 0] == 1


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.mark.gpu
def test_standalone_observations_match_oracle():
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    import torch

    from leviathan_v1_b200 import HubTransitions

    rng = np.random.default_rng(3)
    hubs = [5, 17, 0, 99, 42, 63]
    m = HubTransitions(hubs)
    o = HubCounter(hubs)
    specials = np.array([np.float32(3.1415926), np.nextafter(np.float32(3.1415926),
                         np.float32(4)), -1.0, 7.0, np.nan, 6.2831853, -6.2831853],
                        np.float32)
    for k in range(400):
        th = rng.uniform(-8, 14, 100).astype(np.float32)
        th[rng.integers(0, 100, 3)] = specials[rng.integers(0, len(specials), 3)]
        if k % 2:
            m.accumulate(torch.tensor(th, device="cuda"))
        else:
            m.accumulate(th)
        o.observe(th)
    counts, totals, prev, obs = m.read()
    np.testing.assert_array_equal(counts.astype(np.int64), o.counts)
    np.testing.assert_array_equal(totals.astype(np.int64), o.totals)
    assert prev == o.prev and obs == o.observed == 400
    m.reset()
    counts, totals, prev, obs = m.read()
    assert counts.sum() == 0 and totals.sum() == 0 and prev == -1 and obs == 0
    m.close()


@pytest.mark.gpu
@pytest.mark.parametrize("pairs", [True, False])
def test_engine_observes_every_step(pairs):
    """Attached to an engine, the monitor sees every step (one step per
    launch, or two) and the simulation itself is unchanged."""
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200 import HubTransitions, LeviathanEngine
    from leviathan_v1_b200.graphs import make_network

    net = make_network(5000, 12, 0.1, 20, seed=31)
    hubs = [0, 1, 77, 2500, 4999, 1234, 3001, 4096, 256, 255]
    a = LeviathanEngine(*net.engine_args())
    b = LeviathanEngine(*net.engine_args())
    a.set_pair_mode(pairs)
    m = HubTransitions(hubs)
    m.attach(a)
    o = HubCounter(hubs)
    ra = np.concatenate([a.step_n(DT, 63), [a.step(DT)], a.step_n(DT, 100)])
    rb = []
    for _ in range(164):
        rb.append(b.step(DT))
        o.observe(b.get_theta())
    np.testing.assert_array_equal(ra, np.array(rb, np.float32))
    counts, totals, prev, obs = m.read()
    assert obs == o.observed == 164
    np.testing.assert_array_equal(counts.astype(np.int64), o.counts)
    np.testing.assert_array_equal(totals.astype(np.int64), o.totals)
    assert prev == o.prev
    # detached: no more observations
    m.detach()
    a.step_n(DT, 10)
    assert m.read()[3] == 164
    m.close()
    a.close()
    b.close()


@pytest.mark.gpu
def test_batch_engine_observes_one_network():
    if not has_gpu():
        pytest.fail("needs a CUDA device")
    from leviathan_v1_b200 import BatchEngine, HubTransitions, LeviathanEngine
    from leviathan_v1_b200.graphs import make_network

    nets = [make_network(n, k, 0.1, 16, seed=s) for n, k, s in [(800, 8, 1), (3000, 20, 2)]]
    be = BatchEngine([n.as_dict() for n in nets])
    hubs = [3, 2999, 1500]
    m = HubTransitions(hubs)
    m.attach(be, net=1)
    be.step_n(DT, 40)
    e = LeviathanEngine(*nets[1].engine_args())
    o = HubCounter(hubs)
    for _ in range(40):
        e.step(DT)
        o.observe(e.get_theta())
    counts, totals, prev, obs = m.read()
    np.testing.assert_array_equal(counts.astype(np.int64), o.counts)
    assert obs == 40 and prev == o.prev
    with pytest.raises(ValueError, match="beyond"):
        HubTransitions([900]).attach(be, net=0)
    m.close()
    be.close()
    e.close()
