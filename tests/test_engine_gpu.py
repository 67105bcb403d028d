"""Parity of the B200 engine (CUDA, through the C ABI) with the reference
engine and the FP64 oracle.  Needs a CUDA device.

Tolerances (FP32, stated here and asserted):
* against the reference engine, same inputs, reference math mode, <= 200
  steps: phases within 1e-4 rad (circular distance), weights within 1e-5,
  r within 1e-5 -- and the fraction of bit-identical values is asserted
  separately where the arithmetic is identical;
* against the FP64 oracle over 200 steps: wrapped phase error <= 1e-4 rad in
  accurate math mode;
* integer / index work (ring slots, buf_idx, step count) is exact.
"""

import numpy as np
import pytest

from conftest import (LevAdapter, OracleAdapter, golden_cases, has_gpu,
                      load_golden, network_from_golden, record_from_golden)
from leviathan_v1_b200 import BatchEngine, LeviathanEngine
from leviathan_v1_b200.graphs import make_network
from make_golden import decode_actions, replay
from oracle64 import OracleEngine, circular_distance

pytestmark = pytest.mark.gpu

DT = 0.05
REF_TOL = dict(r=1e-5, theta=1e-4, w=1e-5, hat=1e-4)


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not has_gpu():
        pytest.fail("GPU tests need a CUDA device")


def _cmp(name, got, want, tol, nan_equal=True):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    fin = np.isfinite(want)
    if nan_equal:
        assert np.array_equal(np.isfinite(got), fin), f"{name}: NaN pattern"
    if name.startswith(("theta@", "ring@")):
        err = circular_distance(got[fin], want[fin]).max(initial=0)
    else:
        err = np.abs(got[fin] - want[fin]).max(initial=0)
    assert err <= tol, f"{name}: max error {err} > {tol}"
    return err


# ---------------------------------------------------------------------------
# Reference golden vectors (the reference engine's own outputs)
# ---------------------------------------------------------------------------
@pytest.mark.skipif(not golden_cases(), reason="golden vectors not generated")
@pytest.mark.parametrize("case", golden_cases() or ["none"])
def test_engine_matches_reference_golden(case):
    z = load_golden(case)
    net = network_from_golden(z)
    eng = LevAdapter(net, "reference")
    rs, snaps = replay(eng, decode_actions(z), record_from_golden(z), dt=float(z["dt"]))
    eng.close()
    ref_r = z["r"]
    horizon = min(200, rs.size)
    _cmp("r", rs[:horizon], ref_r[:horizon], REF_TOL["r"])
    for key, got in snaps.items():
        name, t = key.split("@")
        if int(t) > 200:
            continue
        want = z[key]
        if name == "buf_idx":
            assert int(got) == int(want), key
        elif name in ("theta", "ring"):
            _cmp(key, got, want, REF_TOL["theta"])
        elif name == "weights":
            _cmp(key, got, want, REF_TOL["w"])
        elif name in ("theta_hat", "omega_hat"):
            _cmp(key, got, want, REF_TOL["hat"])
        elif name == "g":
            assert abs(float(got) - float(want)) <= 1e-5, key


@pytest.mark.skipif(not golden_cases(), reason="golden vectors not generated")
@pytest.mark.parametrize("case", golden_cases() or ["none"])
def test_engine_bit_identical_to_reference_golden(case):
    """Reference math mode reproduces the reference engine bit for bit
    (same expressions, same intrinsic, same summation order)."""
    z = load_golden(case)
    net = network_from_golden(z)
    eng = LevAdapter(net, "reference")
    rs, snaps = replay(eng, decode_actions(z), record_from_golden(z), dt=float(z["dt"]))
    eng.close()
    np.testing.assert_array_equal(rs, z["r"])
    for key, got in snaps.items():
        np.testing.assert_array_equal(np.asarray(got), z[key], err_msg=key)


def _replay_blocks(e, actions, record, dt):
    """make_golden.replay with every run of steps between two recorded
    points taken as one step block (lev_step_n: graph replay, two steps per
    launch where the network has no zero delay)."""
    rs, out, t = [], {}, 0
    points = sorted(set().union(*record.values()))
    for act in actions:
        kind = act[0]
        if kind == "step":
            end = t + act[1]
            while t < end:
                nxt = min([p for p in points if t < p <= end] or [end])
                rs.append(e.step_n(dt, nxt - t))
                t = nxt
                if t in points:
                    th_hat, om_hat = e.get_predictor()
                    ring, bi = e.get_ring(0)
                    snap = dict(theta=e.get_theta(), weights=e.get_weights(),
                                theta_hat=th_hat, omega_hat=om_hat, ring=ring,
                                buf_idx=np.int32(bi))
                    for key, names in (("theta", ["theta"]), ("weights", ["weights"]),
                                       ("predictor", ["theta_hat", "omega_hat"]),
                                       ("ring", ["ring", "buf_idx"])):
                        if t in record.get(key, ()):
                            for nm in names:
                                out[f"{nm}@{t}"] = snap[nm]
                    out[f"g@{t}"] = np.float32(e.get_gain())
        elif kind == "set_theta":
            th = e.get_theta()
            e.set_theta(((th + act[1]) % np.float32(2 * np.pi)).astype(np.float32))
        elif kind == "set_theta_raw":
            th = e.get_theta().copy()
            m = act[1] != 0
            th[m] = act[1][m]
            e.set_theta(th.astype(np.float32))
        elif kind == "set_gain":
            e.set_gain(act[1])
        elif kind == "controller":
            e.set_gain_controller(act[1])
    return np.concatenate(rs).astype(np.float32), out


@pytest.mark.skipif(not golden_cases(), reason="golden vectors not generated")
@pytest.mark.parametrize("case", golden_cases() or ["none"])
@pytest.mark.parametrize("path", ["graph", "cluster", "grid"])
def test_step_blocks_bit_identical_to_reference_golden(case, path):
    """Step blocks (graph replay with two steps per launch where no delay is
    0, the cluster-resident kernel, the grid-resident kernel) reproduce the
    reference engine bit for bit, including blocks of odd length and blocks
    interrupted by set_theta / gain / controller calls."""
    z = load_golden(case)
    net = network_from_golden(z)
    e = LeviathanEngine(*net.engine_args())
    e.set_cluster_mode(path == "cluster")
    e.set_grid_mode(path == "grid")
    if path == "cluster" and not e.cluster_info()["eligible"]:
        e.close()
        pytest.skip("cluster path not eligible")
    if path == "grid" and not e.grid_info()["eligible"]:
        e.close()
        pytest.skip("grid path not eligible")
    assert e.pair_info()[0]["eligible"] == bool(np.all(net.delays > 0))
    rs, snaps = _replay_blocks(e, decode_actions(z), record_from_golden(z), float(z["dt"]))
    e.close()
    np.testing.assert_array_equal(rs, z["r"])
    for key, got in snaps.items():
        np.testing.assert_array_equal(np.asarray(got), z[key], err_msg=key)


def test_division_free_wraps_are_bitwise_ieee_for_all_inputs():
    """The phase wraps evaluated without a division equal the reference's
    IEEE-division expressions (leviathan_kernel.cu:105,146,188) in every bit,
    for all 2^32 float inputs."""
    import ctypes as C

    from leviathan_v1_b200 import _lib

    lib = _lib.load()
    a, b = C.c_uint64(), C.c_uint64()
    assert lib.lev_selftest_wraps(C.byref(a), C.byref(b)) == 0
    assert a.value == 0 and b.value == 0, (a.value, b.value)


# ---------------------------------------------------------------------------
# Live reference engine (oracle/_ref) on larger inputs
# ---------------------------------------------------------------------------
def _ref_engine(net, flavor="sm100a"):
    from refengine import RefEngine, available

    if not available(flavor):
        pytest.fail("oracle/_ref/ reference build missing (run make -C oracle)")
    return RefEngine(*net.engine_args(), flavor=flavor)


@pytest.mark.parametrize("blocks", [False, True], ids=["step", "step_n"])
@pytest.mark.parametrize("N,k,md,steps", [(20_000, 16, 30, 60), (100_000, 32, 64, 20),
                                          (1_000_000, 32, 64, 6),
                                          (50_000, 16, 255, 300)])  # largest delay; ring wraps
def test_engine_matches_live_reference(N, k, md, steps, blocks):
    """Against the reference engine itself on the same GPU; ``step_n``
    takes two steps per launch (pair and finish kernels)."""
    net = make_network(N, k, 0.1, md, seed=N)
    ref = _ref_engine(net)
    eng = LeviathanEngine(*net.engine_args())
    r_ref = ref.run(DT, steps)
    if blocks:
        assert eng.pair_info()[0]["eligible"]
        r_eng = eng.step_n(DT, steps)
    else:
        r_eng = np.array([eng.step(DT) for _ in range(steps)], np.float32)
    s = ref.state()
    _cmp("r", r_eng, r_ref, REF_TOL["r"])
    _cmp("theta@", eng.get_theta(), s["theta"], REF_TOL["theta"])
    _cmp("weights", eng.get_weights(), s["weights"], REF_TOL["w"])
    ring, bi = eng.get_ring(0)
    assert bi == s["buf_idx"] == steps % (md + 1)
    _cmp("ring@", ring, s["ring"], REF_TOL["theta"])
    assert abs(eng.get_gain() - s["g"]) <= 1e-5
    same = np.mean(eng.get_theta() == s["theta"])
    assert same > 0.999, f"only {same:.4%} of phases bit-identical"
    ref.close()
    eng.close()


def test_stock_reference_build_agrees():
    """The reference's stock arch list (PTX JIT on B200) runs and agrees."""
    net = make_network(5000, 16, 0.1, 20, seed=9)
    a = _ref_engine(net, "sm100a")
    b = _ref_engine(net, "stock")
    ra, rb = a.run(DT, 30), b.run(DT, 30)
    _cmp("r", ra, rb, REF_TOL["r"])
    a.close()
    b.close()


# ---------------------------------------------------------------------------
# FP64 oracle
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("mode,tol", [("accurate", 1e-4), ("reference", 2e-3)])
def test_error_against_fp64_oracle(mode, tol):
    net = make_network(1000, 20, 0.1, 50, seed=0, generator="networkx")
    eng = LeviathanEngine(*net.engine_args(), math_mode=mode)
    o = OracleEngine(*net.engine_args())
    r_eng = eng.step_n(DT, 200)
    r_o = o.run(DT, 200)
    err = circular_distance(eng.get_theta(), o.theta).max()
    assert err <= tol, f"{mode}: wrapped phase error {err}"
    assert np.abs(r_eng - r_o).max() <= 10 * tol
    eng.close()


def _degenerate(kind):
    from leviathan_v1_b200.graphs import Network, init_state

    if kind == "no_edges":          # every row empty
        N, md, rp, col = 777, 9, np.zeros(778, np.int32), np.zeros(0, np.int32)
    elif kind == "one_node":        # a single node coupled to itself
        N, md, rp, col = 1, 3, np.array([0, 1], np.int32), np.zeros(1, np.int32)
    elif kind == "one_node_no_edge":
        N, md, rp, col = 1, 0, np.zeros(2, np.int32), np.zeros(0, np.int32)
    else:                           # 33 rows: one full slice and one row more
        N, md = 33, 5
        deg = np.arange(N) % 4
        rp = np.zeros(N + 1, np.int32)
        np.cumsum(deg, out=rp[1:])
        col = (np.repeat(np.arange(N), deg) + np.concatenate(
            [np.arange(1, d + 1) for d in deg])) % N
        col = col.astype(np.int32)
    st = init_state(rp, md, 5, delay_lo=min(1, md))
    return Network(N, md, rp, col, st["delays"], st["weights"], st["theta"],
                   st["theta_hat"], st["omega"])


@pytest.mark.parametrize("kind", ["no_edges", "one_node", "one_node_no_edge", "ragged_33"])
def test_degenerate_networks_match_fp64_oracle(kind):
    """Empty edge lists, a single node, and a row count just past one slice,
    against the FP64 oracle, by single steps and by step blocks."""
    net = _degenerate(kind)
    o = OracleEngine(*net.engine_args())
    r_o = o.run(DT, 60)
    for blocks in (False, True):
        eng = LeviathanEngine(*net.engine_args(), math_mode="accurate")
        if blocks:
            r = eng.step_n(DT, 60)
        else:
            r = np.array([eng.step(DT) for _ in range(60)], np.float32)
        assert np.abs(r - r_o).max() <= 1e-4, (kind, blocks)
        assert circular_distance(eng.get_theta(), o.theta).max() <= 1e-4, (kind, blocks)
        if net.E:
            assert np.abs(eng.get_weights() - o.w).max() <= 1e-5, (kind, blocks)
        assert eng.step_count() == 60
        eng.close()


# ---------------------------------------------------------------------------
# Engine properties
# ---------------------------------------------------------------------------
def test_step_n_equals_repeated_step():
    net = make_network(3000, 12, 0.1, 25, seed=4)
    a = LeviathanEngine(*net.engine_args())
    b = LeviathanEngine(*net.engine_args())
    ra = np.array([a.step(DT) for _ in range(300)], np.float32)
    rb = np.concatenate([b.step_n(DT, 7), b.step_n(DT, 256), b.step_n(DT, 37)])
    np.testing.assert_array_equal(ra, rb)
    np.testing.assert_array_equal(a.get_theta(), b.get_theta())
    np.testing.assert_array_equal(a.get_weights(), b.get_weights())
    assert a.step_count() == b.step_count() == 300


def test_block_issued_directly_then_recorded_then_replayed():
    """The first block of a length is issued directly, the second records a
    CUDA graph, the third replays it: all three equal single steps."""
    net = make_network(30_000, 16, 0.1, 20, seed=12)
    a = LeviathanEngine(*net.engine_args())
    b = LeviathanEngine(*net.engine_args())
    for eng in (a, b):
        eng.set_cluster_mode(False)
        eng.set_grid_mode(False)
    ra = np.array([a.step(DT) for _ in range(3 * 24)], np.float32)
    rb = np.concatenate([b.step_n(DT, 24) for _ in range(3)])
    np.testing.assert_array_equal(ra, rb)
    np.testing.assert_array_equal(a.get_theta(), b.get_theta())
    np.testing.assert_array_equal(a.get_weights(), b.get_weights())
    a.close()
    b.close()


@pytest.mark.parametrize("batch", [False, True])
def test_speculative_single_steps_bit_identical(batch):
    """Single steps run as speculative pairs (the pair kernel's second walk
    into shadow buffers, finished by the next call): after every call the
    engine state equals that of plain one-step blocks, bit for bit, with the
    state read back and written (theta, weights, gain, controller,
    parameters, dt) between calls."""
    nets = [make_network(20_000, 16, 0.1, 30, seed=31)]
    if batch:
        nets += [make_network(3000, 12, 0.1, 20, seed=32)]

    def make():
        if batch:
            return BatchEngine([n.as_dict() for n in nets])
        return LeviathanEngine(*nets[0].engine_args())

    a, b = make(), make()
    for e in (a, b):
        e.set_cluster_mode(False)
        e.set_grid_mode(False)
    assert all(c["enabled"] for c in a.pair_info() if c["eligible"])
    rng = np.random.default_rng(5)
    dt = DT
    for k in range(40):
        ra = a._step_all(dt)
        rb = b._step_n_all(dt, 1)[0]
        np.testing.assert_array_equal(ra, rb, err_msg=f"step {k}")
        if k % 3 == 0:
            sa, sb = _full_state(a), _full_state(b)
            for key, want in sb.items():
                np.testing.assert_array_equal(sa[key], want, err_msg=f"step {k}: {key}")
        if k == 10:
            for e in (a, b):
                e._set_gain(0.7, 0)
        if k == 14:
            for e in (a, b):
                e._set_ctrl(False, 0)
        if k == 19:
            th = rng.uniform(0, 2 * np.pi, a.total_nodes).astype(np.float32)
            for e in (a, b):
                e.set_all_theta(th)
        if k == 25:
            dt = 0.04
        if k == 31:
            for e in (a, b):
                e._set_ctrl(True, 0)
                e.set_params(0, eta=0.02) if batch else e.set_params(eta=0.02)
    sa, sb = _full_state(a), _full_state(b)
    for key, want in sb.items():
        np.testing.assert_array_equal(sa[key], want, err_msg=key)
    a.close()
    b.close()


def test_batch_equals_individual_engines():
    nets = [make_network(n, k, 0.1, md, seed=s, delay_lo=min(1, md))
            for n, k, md, s in [(700, 8, 10, 1), (2500, 20, 50, 2), (256, 4, 3, 3),
                                (1000, 16, 0, 4), (4097, 32, 64, 5)]]
    params = [dict(g=0.5 * i, gain_controller=i % 2) for i in range(len(nets))]
    be = BatchEngine([n.as_dict() for n in nets], params=params)
    rb = be.step_n(DT, 120)
    for i, n in enumerate(nets):
        e = LeviathanEngine(*n.engine_args(), params=params[i])
        ri = e.step_n(DT, 120)
        np.testing.assert_array_equal(rb[:, i], ri)
        np.testing.assert_array_equal(be.get_theta(i), e.get_theta())
        e.close()
    be.close()


def test_batch_with_an_edgeless_network():
    """A network without edges between two with edges: the device packing
    writes nothing for it and the neighbours' slices stay in place."""
    from leviathan_v1_b200.graphs import Network, init_state

    a = make_network(900, 8, 0.1, 12, seed=7)
    rp = np.zeros(301, np.int32)
    st = init_state(rp, 5, 9)
    empty = Network(300, 5, rp, np.zeros(0, np.int32), st["delays"], st["weights"],
                    st["theta"], st["theta_hat"], st["omega"])
    c = make_network(1500, 12, 0.1, 20, seed=8)
    nets = [a, empty, c]
    be = BatchEngine([n.as_dict() for n in nets])
    rb = be.step_n(DT, 40)
    for i, n in enumerate(nets):
        e = LeviathanEngine(*n.engine_args())
        np.testing.assert_array_equal(rb[:, i], e.step_n(DT, 40))
        np.testing.assert_array_equal(be.get_theta(i), e.get_theta())
        e.close()
    be.close()


@pytest.mark.parametrize("N,k,md,ctrl", [(1000, 20, 50, 1), (700, 8, 10, 0),
                                         (4096, 32, 64, 1), (3000, 12, 0, 1),
                                         (16000, 8, 8, 1)])
def test_cluster_path_bit_identical(N, k, md, ctrl):
    """The cluster-resident kernel (whole network in the shared memory of one
    thread-block cluster, many steps per launch) gives bitwise the results of
    the per-step kernel."""
    net = make_network(N, k, 0.1, md, seed=N + md, delay_lo=min(1, md))
    a = LeviathanEngine(*net.engine_args(), params=dict(gain_controller=ctrl))
    b = LeviathanEngine(*net.engine_args(), params=dict(gain_controller=ctrl))
    info = a.cluster_info()
    assert info["eligible"], info
    a.set_cluster_mode(True)
    b.set_cluster_mode(False)
    b.set_grid_mode(False)
    ra = np.concatenate([a.step_n(DT, 5), a.step_n(DT, 300)])
    rb = np.concatenate([b.step_n(DT, 5), b.step_n(DT, 300)])
    np.testing.assert_array_equal(ra, rb)
    np.testing.assert_array_equal(a.get_theta(), b.get_theta())
    np.testing.assert_array_equal(a.get_weights(), b.get_weights())
    ga, gb = a.get_predictor(), b.get_predictor()
    np.testing.assert_array_equal(ga[0], gb[0])
    np.testing.assert_array_equal(ga[1], gb[1])
    assert a.get_gain() == b.get_gain() and a.step_count() == b.step_count() == 305
    ring_a, bi_a = a.get_ring()
    ring_b, bi_b = b.get_ring()
    assert bi_a == bi_b
    np.testing.assert_array_equal(ring_a, ring_b)
    # and a single step after the block still continues identically
    assert a.step(DT) == b.step(DT)
    a.close()
    b.close()


@pytest.mark.parametrize("N,k,md,ctrl,mode", [(10_000, 20, 50, 1, "reference"),
                                              (10_000, 20, 50, 1, "accurate"),
                                              (3000, 12, 0, 1, "reference"),
                                              (20_000, 32, 64, 0, "reference"),
                                              (1000, 20, 50, 1, "reference"),
                                              (4097, 8, 5, 1, "reference")])
def test_grid_path_bit_identical(N, k, md, ctrl, mode):
    """The grid-resident kernel (one cooperative launch per step block, a grid
    barrier per step) gives bitwise the results of the per-step kernel, for
    every eligible rows-per-CTA choice, zero delays included."""
    net = make_network(N, k, 0.1, md, seed=N + md + 3, delay_lo=min(1, md))
    b = LeviathanEngine(*net.engine_args(), params=dict(gain_controller=ctrl), math_mode=mode)
    b.set_cluster_mode(False)
    b.set_grid_mode(False)
    rb = np.concatenate([b.step_n(DT, 5), b.step_n(DT, 300)])
    want = _full_state(b)
    rb_next = b.step(DT)
    b.close()
    probe = LeviathanEngine(*net.engine_args(), math_mode=mode)
    info = probe.grid_info()
    probe.close()
    assert info["eligible"] and info["eligible_rows"], info
    for R in info["eligible_rows"]:
        a = LeviathanEngine(*net.engine_args(), params=dict(gain_controller=ctrl),
                            math_mode=mode)
        a.set_cluster_mode(False)
        a.set_grid_mode(True, R)
        assert a.grid_info()["rows_per_cta"] == R
        ra = np.concatenate([a.step_n(DT, 5), a.step_n(DT, 300)])
        np.testing.assert_array_equal(ra, rb, err_msg=f"R={R}")
        got = _full_state(a)
        for key, w in want.items():
            np.testing.assert_array_equal(got[key], w, err_msg=f"R={R}: {key}")
        assert a.step(DT) == rb_next
        a.close()


def test_grid_path_not_used_when_too_large():
    net = make_network(200_000, 8, 0.1, 8, seed=2)
    e = LeviathanEngine(*net.engine_args())
    assert not e.grid_info()["eligible"]
    e.close()


def test_cluster_path_not_used_when_too_large():
    net = make_network(40_000, 16, 0.1, 20, seed=1)
    e = LeviathanEngine(*net.engine_args())
    assert not e.cluster_info()["eligible"]
    e.close()


def test_autotune_leaves_simulation_unchanged():
    nets = [make_network(n, k, 0.1, 20, seed=s)
            for n, k, s in [(3000, 8, 1), (2000, 20, 2), (5000, 32, 3)]]
    a = BatchEngine([n.as_dict() for n in nets])
    b = BatchEngine([n.as_dict() for n in nets])
    classes = [c for c in a.tuning() if c["tiles"]]
    assert len(classes) == 3  # k = 8, 20, 32 fall in three degree classes
    ra = [a.step_n(DT, 20)]
    res = a.autotune(DT, trial_steps=3)
    assert all(0 <= v < len(res["variants"]) for v in res["chosen"])
    ra.append(a.step_n(DT, 30))
    rb = b.step_n(DT, 50)
    np.testing.assert_array_equal(np.concatenate(ra), rb)
    np.testing.assert_array_equal(a.get_theta(), b.get_theta())
    np.testing.assert_array_equal(a.get_weights(), b.get_weights())
    for c in range(3):  # every variant gives the same bits
        for v in range(len(res["variants"])):
            b.set_variant(c, v)
            a.set_variant(c, (v + 1) % len(res["variants"]))
            np.testing.assert_array_equal(a.step_n(DT, 2), b.step_n(DT, 2))
    a.close()
    b.close()


def _full_state(e):
    th_hat, om_hat = e.get_predictor()
    out = dict(theta=e.get_all_theta(), weights=e.get_weights(), theta_hat=th_hat,
               omega_hat=om_hat)
    for k in range(e.num_nets):
        ring, bi = e.get_ring(k)
        out[f"ring{k}"] = ring
        out[f"buf{k}"] = np.int64(bi)
        out[f"g{k}"] = np.float32(e._get_gain(k))
        out[f"t{k}"] = np.int64(e.step_count(k))
    return out


@pytest.mark.parametrize("mode", ["reference", "accurate"])
def test_two_steps_per_launch_bit_identical(mode):
    """Two steps per launch (pair_kernel + finish_kernel) against one step
    per launch: every pair variant, a single network at scale and a batch of
    uneven networks, odd block lengths, controller on and off."""
    from leviathan_v1_b200 import _lib
    from leviathan_v1_b200.engine import pair_variant_info

    nvar = _lib.load().lev_num_pair_variants()
    assert any(pair_variant_info(v)["deep"] for v in range(nvar))
    single = make_network(20_000, 16, 0.1, 30, seed=77)
    batch = [make_network(n, k, 0.1, md, seed=s)
             for n, k, md, s in [(700, 8, 10, 1), (2500, 20, 50, 2), (300, 4, 3, 3),
                                 (4097, 32, 64, 5), (1500, 12, 1, 6)]]
    params = [dict(g=0.4 * i, gain_controller=i % 2) for i in range(len(batch))]
    for make in (lambda: LeviathanEngine(*single.engine_args(), math_mode=mode),
                 lambda: BatchEngine([n.as_dict() for n in batch], params=params,
                                     math_mode=mode)):
        ref = make()
        ref.set_cluster_mode(False)
        ref.set_grid_mode(False)
        ref.set_pair_mode(False)
        assert not any(c["enabled"] for c in ref.pair_info())
        r_ref = np.concatenate([ref.step_n(DT, 3), ref.step_n(DT, 64), ref.step_n(DT, 13)])
        s_ref = _full_state(ref)
        ref.close()
        for v in range(nvar):
            e = make()
            e.set_cluster_mode(False)
            e.set_grid_mode(False)
            for c in range(3):
                e.set_pair_variant(c, v)
            info = e.pair_info()
            assert all(c["eligible"] and c["enabled"] for c in info), info
            r = np.concatenate([e.step_n(DT, 3), e.step_n(DT, 64), e.step_n(DT, 13)])
            np.testing.assert_array_equal(r, r_ref, err_msg=f"pair variant {v}")
            for key, want in s_ref.items():
                np.testing.assert_array_equal(_full_state(e)[key], want,
                                              err_msg=f"pair variant {v}: {key}")
            e.close()


def test_zero_delay_takes_one_step_per_launch():
    """A zero delay reads theta_j(t+1) in step t+1, which another CTA writes
    in the same launch: such engines are not eligible and step blocks take
    one step per launch (still equal to repeated single steps)."""
    net = make_network(3000, 12, 0.1, 6, seed=12, delay_lo=0)
    assert (net.delays == 0).any()
    a = LeviathanEngine(*net.engine_args())
    b = LeviathanEngine(*net.engine_args())
    a.set_cluster_mode(False)
    a.set_grid_mode(False)
    info = a.pair_info()
    assert not info[0]["eligible"] and not info[0]["enabled"]
    ra = a.step_n(DT, 41)
    rb = np.array([b.step(DT) for _ in range(41)], np.float32)
    np.testing.assert_array_equal(ra, rb)
    np.testing.assert_array_equal(a.get_theta(), b.get_theta())
    a.close()
    b.close()


def test_checkpoint_round_trip_is_exact():
    net = make_network(5000, 16, 0.1, 40, seed=8)
    e = LeviathanEngine(*net.engine_args())
    e.step_n(DT, 25)
    st = e.get_state()
    r1 = e.step_n(DT, 60)
    th1 = e.get_theta()
    e.set_state(st)
    r2 = e.step_n(DT, 60)
    np.testing.assert_array_equal(r1, r2)
    np.testing.assert_array_equal(th1, e.get_theta())
    e.close()


def test_set_theta_refills_ring_and_resets_history():
    net = make_network(2000, 10, 0.1, 15, seed=2)
    e = LeviathanEngine(*net.engine_args())
    e.step_n(DT, 33)
    th = np.linspace(0, 6.0, 2000).astype(np.float32)
    e.set_theta(th)
    ring, bi = e.get_ring()
    assert bi == 33 % 16
    np.testing.assert_array_equal(ring, np.repeat(th[:, None], 16, axis=1))
    with pytest.raises(RuntimeError, match="size mismatch"):
        e.set_theta(th[:10])
    e.close()


def test_invariants_at_scale():
    net = make_network(1_000_000, 32, 0.1, 64, seed=0)
    e = LeviathanEngine(*net.engine_args())
    r = e.step_n(DT, 50)
    th = e.get_theta()
    w = e.get_weights()
    assert np.all(np.isfinite(th)) and th.min() >= 0 and th.max() < 2 * np.pi + 1e-5
    assert np.all((r >= 0) & (r <= 1))
    assert w.min() >= 0 and w.max() <= 2
    assert e.step_count() == 50
    e.close()


@pytest.mark.parametrize("N,k,p", [(5000, 10, 0.1), (100_000, 32, 0.1), (2000, 8, 0.0),
                                   (300, 20, 1.0)])
def test_gpu_graph_generator(N, k, p):
    from leviathan_v1_b200.graphs import make_network_gpu

    a = make_network_gpu(N, k, p, 50, seed=7)
    b = make_network_gpu(N, k, p, 50, seed=7)
    c = make_network_gpu(N, k, p, 50, seed=8)
    rp, col = a.row_ptr, a.col_idx
    assert rp[0] == 0 and rp[-1] == N * k and np.all(np.diff(rp) >= 0)
    rows = np.repeat(np.arange(N), np.diff(rp))
    assert np.all((col >= 0) & (col < N)) and not np.any(rows == col)
    key = rows.astype(np.int64) * N + col
    assert np.all(np.diff(key) > 0)  # sorted, no multi-edges
    assert np.array_equal(np.sort(key), np.sort(col.astype(np.int64) * N + rows))  # symmetric
    for x, y in zip(a.engine_args()[2:], b.engine_args()[2:]):
        np.testing.assert_array_equal(x, y)  # deterministic
    if p > 0:
        assert not np.array_equal(a.col_idx, c.col_idx)
        d = np.abs(rows - col)
        far = np.mean(np.minimum(d, N - d) > k // 2)
        assert abs(far - p) < 0.02 + 0.1 * p * (N < 1000)
    else:
        d = np.abs(rows - col)
        assert np.all(np.minimum(d, N - d) <= k // 2)
    assert a.delays.min() >= 1 and a.delays.max() <= 50
    assert np.all((a.weights >= 0) & (a.weights < 1))
    assert np.all((a.theta >= 0) & (a.theta <= np.float32(2 * np.pi)))
    if N >= 5000:
        assert abs(float(a.omega.mean())) < 0.1 and abs(float(a.omega.std()) - 1) < 0.1
    e = LeviathanEngine(*a.engine_args())
    assert np.all(np.isfinite(e.step_n(DT, 20)))
    e.close()


def test_invalid_topology_rejected_on_device():
    net = make_network(500, 8, 0.1, 10, seed=1)
    col = net.col_idx.copy()
    col[17] = 500
    with pytest.raises(ValueError, match="col_idx"):
        LeviathanEngine(net.N, 10, net.row_ptr, col, net.delays, net.weights,
                        net.theta, net.theta_hat, net.omega)
    col[17] = -3
    with pytest.raises(ValueError, match="col_idx"):
        LeviathanEngine(net.N, 10, net.row_ptr, col, net.delays, net.weights,
                        net.theta, net.theta_hat, net.omega)
    d = net.delays.copy()
    d[3] = 11
    with pytest.raises(ValueError, match="delay"):
        LeviathanEngine(net.N, 10, net.row_ptr, net.col_idx, d, net.weights,
                        net.theta, net.theta_hat, net.omega)
    # in a batch, each network's columns are checked against its own N
    small = make_network(300, 8, 0.1, 10, seed=2)
    bad = small.as_dict()
    bad["col_idx"] = bad["col_idx"].copy()
    bad["col_idx"][-1] = 300  # valid in the first network (N = 500), not here
    with pytest.raises(ValueError, match="col_idx"):
        BatchEngine([net.as_dict(), bad])


def test_invalid_row_ptr_and_sizes_rejected():
    """Shape errors found by the host layout pass, which runs while the edge
    arrays are already on their way to the device: each creation fails with
    its message, releases what it took, and the next engine is fine."""
    net = make_network(2000, 8, 0.1, 10, seed=3)
    args = list(net.engine_args())
    rp = net.row_ptr.copy()
    rp[700] = rp[699] - 1  # decreasing at row 699
    with pytest.raises(ValueError, match="decreasing at row 699"):
        LeviathanEngine(*(args[:2] + [rp] + args[3:]))
    rp = net.row_ptr.copy()
    rp[0] = 1
    with pytest.raises(ValueError, match="row_ptr\\[0\\]"):
        LeviathanEngine(*(args[:2] + [rp] + args[3:]))
    with pytest.raises(ValueError, match="max_delay"):
        LeviathanEngine(*([net.N, 256] + args[2:]))
    e = LeviathanEngine(*args)
    ref = LeviathanEngine(*args)
    np.testing.assert_array_equal(e.step_n(DT, 20), ref.step_n(DT, 20))
    e.close()
    ref.close()


def test_reference_abi_layer():
    """The reference's C ABI on this library behaves like the Python class."""
    import ctypes as C

    from leviathan_v1_b200 import _lib

    lib = _lib.load()
    net = make_network(800, 8, 0.1, 12, seed=6)
    arrs = [np.ascontiguousarray(a) for a in net.engine_args()[2:]]
    P = lambda a: C.c_void_p(a.ctypes.data)
    h = lib.leviathan_init(net.N, net.max_delay, *[P(a) for a in arrs])
    assert h
    e = LeviathanEngine(*net.engine_args())
    for _ in range(20):
        assert lib.leviathan_step(h, C.c_float(DT)) == np.float32(e.step(DT))
    th = np.empty(net.N, np.float32)
    lib.leviathan_get_theta(h, P(th))
    np.testing.assert_array_equal(th, e.get_theta())
    lib.leviathan_set_gain(h, C.c_float(2.0))
    assert lib.leviathan_get_gain(h) == np.float32(2.0)
    assert lib.leviathan_get_vram_usage(h) > 0
    lib.leviathan_free(h)
    e.close()


def test_engine_memory_pool_and_creation_profile():
    """Engines take their device memory from the library's pool: a freed
    engine's memory serves the next one; lev_trim_memory returns it to the
    device, and engines still work afterwards.  The creation profile names
    every phase with a non-negative time."""
    from leviathan_v1_b200 import _lib

    lib = _lib.load()
    net = make_network(20_000, 16, 0.1, 30, seed=31)
    a = LeviathanEngine(*net.engine_args())
    prof = a.create_profile()
    assert len(prof) == 8 and all(v >= 0.0 for v in prof.values())
    ra = a.step_n(DT, 30)
    a.close()
    b = LeviathanEngine(*net.engine_args())  # reuses the pooled memory
    np.testing.assert_array_equal(b.step_n(DT, 30), ra)
    b.close()
    assert lib.lev_trim_memory() == 0
    c = LeviathanEngine(*net.engine_args())
    np.testing.assert_array_equal(c.step_n(DT, 30), ra)
    c.close()
