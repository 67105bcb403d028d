"""Long-horizon statistical parity with the reference engine (GPU).

Over at most 200 steps the engine is compared with the reference engine
value by value (test_engine_gpu.py).  The dynamics are chaotic, though: two
FP32 runs that differ in one rounding decorrelate microscopically after
enough steps, so over long horizons agreement is judged on statistics of the
run, as the reference step (leviathan_kernel.cu:391-438, r :237-264) would
be judged against itself:

* time-averaged r over four windows of 500 steps of a 2000-step run (the
  benchmark horizon) and over the whole run;
* the final weight distribution: L1 distance of the 40-bin histograms over
  [w_min, w_max] = [0, 2], and the Kolmogorov-Smirnov distance of the two
  empirical distributions (400-bin grid);
* for the coupling sweep, r(K): the mean r of the last 100 of 1000 steps of
  each network at its fixed K (experiments/phase_sweep.py:25-59), batched
  engine against one reference engine per network, on 16 networks.

Tolerance, per statistic: our engine must be within max(3 s, floor) of the
reference engine, where s is the same statistic's distance between the
reference engine and itself started from phases moved by one float32 ulp
(the size of one rounding difference) -- the engine may differ from the
reference no more than the reference differs from itself -- and the floors
are: window means 0.02 at N = 1000 and 0.005 at N = 10^6, histogram L1 0.02,
KS 0.02, r(K) 0.03 per network (the reference's own scatter over 100 steps
of a 500-node network is of that order).
"""

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

DT = 0.05
STEPS = 2000
WINDOW = 500
BINS = np.linspace(0.0, 2.0, 41)
KS_GRID = np.linspace(0.0, 2.0, 401)


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not has_gpu():
        pytest.fail("GPU tests need a CUDA device")


def _refengine():
    import refengine

    if not refengine.available("sm100a"):
        pytest.skip("reference engine not built (make -C oracle)")
    return refengine


def run_reference(net, steps, theta0=None):
    ref = _refengine().RefEngine(*net.engine_args())
    if theta0 is not None:
        ref.set_theta(theta0)  # every ring slot := theta0, as at init
    r = ref.run(DT, steps)
    w = ref.state()["weights"]
    ref.close()
    return r, w


def run_ours(net, steps, math_mode):
    from leviathan_v1_b200 import LeviathanEngine

    e = LeviathanEngine(*net.engine_args(), math_mode=math_mode)
    r = e.step_n(DT, steps)
    w = e.get_weights()
    e.close()
    return r, w


def stats(r, w):
    r = np.asarray(r, np.float64)
    win = r[: len(r) // WINDOW * WINDOW].reshape(-1, WINDOW).mean(axis=1)
    h = np.histogram(w, BINS)[0] / max(w.size, 1)
    cdf = np.searchsorted(np.sort(w), KS_GRID, side="right") / max(w.size, 1)
    return dict(windows=win, mean=r.mean(), hist=h, cdf=cdf)


def distance(a, b):
    return dict(windows=float(np.abs(a["windows"] - b["windows"]).max()),
                mean=float(abs(a["mean"] - b["mean"])),
                hist_l1=float(np.abs(a["hist"] - b["hist"]).sum()),
                ks=float(np.abs(a["cdf"] - b["cdf"]).max()))


def check_against_reference(net, math_modes, floor_window):
    r_ref, w_ref = run_reference(net, STEPS)
    theta_ulp = np.nextafter(net.theta.astype(np.float32), np.float32(10.0))
    r_pert, w_pert = run_reference(net, STEPS, theta_ulp)
    s_ref = stats(r_ref, w_ref)
    spread = distance(stats(r_pert, w_pert), s_ref)
    floors = dict(windows=floor_window, mean=floor_window, hist_l1=0.02, ks=0.02)
    tol = {k: max(3 * spread[k], floors[k]) for k in floors}
    report = {"spread": spread, "tol": tol}
    for mode in math_modes:
        r, w = run_ours(net, STEPS, mode)
        assert np.all(np.isfinite(r)) and np.all((r >= 0) & (r <= 1))
        d = distance(stats(r, w), s_ref)
        report[mode] = d
        for k in tol:
            assert d[k] <= tol[k], (mode, k, report)
    return report


def test_long_horizon_small_both_math_modes():
    """N = 1000, k = 20, 2000 steps, controller on."""
    from leviathan_v1_b200.graphs import config_small

    rep = check_against_reference(config_small(0), ("reference", "accurate"), 0.02)
    print("long horizon N=1000:", rep)


def test_long_horizon_at_scale():
    """N = 10^6, k = 32, delays [1, 64], 2000 steps, controller on."""
    from leviathan_v1_b200.graphs import config_scale

    rep = check_against_reference(config_scale(0), ("reference", "accurate"), 0.005)
    print("long horizon N=1e6:", rep)


def test_sweep_r_of_K_matches_reference_engines():
    """r(K) of 16 networks of the 512-network sweep (controller off, fixed
    K), batched engine against one reference engine per network."""
    from leviathan_v1_b200 import BatchEngine
    from leviathan_v1_b200.graphs import batch_specs, build_batch

    specs = batch_specs(512, seed=0)
    pick = [specs[i] for i in range(0, 512, 32)]  # 16 networks, K spread over [0, 4]
    nets, params = build_batch(pick)
    eng = BatchEngine([n.as_dict() for n in nets], params=params)
    r = eng.step_n(DT, 1000)
    eng.close()
    ours = r[-100:].mean(axis=0)
    ref, pert = [], []
    for n, p in zip(nets, params):
        for theta0, out in ((None, ref), (np.nextafter(n.theta, np.float32(10.0)), pert)):
            e = _refengine().RefEngine(*n.engine_args())
            e.set_gain_controller(False)
            e.set_gain(p["g"])
            if theta0 is not None:
                e.set_theta(theta0)
            out.append(e.run(DT, 1000)[-100:].mean())
            e.close()
    ref, pert = np.array(ref), np.array(pert)
    tol = np.maximum(3 * np.abs(pert - ref), 0.03)
    print("r(K) ours", ours, "ref", ref, "ref-perturbed", pert)
    assert np.all(np.abs(ours - ref) <= tol), (ours, ref, tol)
    # the curve as a whole: same shape
    assert np.corrcoef(ours, ref)[0, 1] > 0.95
