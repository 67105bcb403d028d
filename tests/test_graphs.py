"""Topology and initial-state generators (CPU)."""

import numpy as np
import pytest

from leviathan_v1_b200.graphs import (config_batch, config_small, init_state,
                                      ws_csr, ws_csr_networkx)


def _check_csr(rp, col, N, k):
    assert rp.dtype == np.int32 and col.dtype == np.int32
    assert rp.shape == (N + 1,) and rp[0] == 0
    assert np.all(np.diff(rp) >= 0)
    assert rp[-1] == N * k  # rewiring moves edges, never adds or drops them
    rows = np.repeat(np.arange(N), np.diff(rp))
    assert np.all(col >= 0) and np.all(col < N)
    assert not np.any(rows == col), "self loop"
    key = rows.astype(np.int64) * N + col
    assert np.all(np.diff(key) > 0), "columns not strictly sorted per row"
    tkey = np.sort(col.astype(np.int64) * N + rows)
    assert np.array_equal(np.sort(key), tkey), "not symmetric"


@pytest.mark.parametrize("N,k,p", [(2000, 10, 0.1), (500, 32, 0.3), (64, 4, 0.0)])
def test_ws_csr_invariants(N, k, p):
    rp, col = ws_csr(N, k, p, seed=3)
    _check_csr(rp, col, N, k)


def test_ws_csr_lattice_at_p0():
    N, k = 50, 6
    rp, col = ws_csr(N, k, 0.0, seed=0)
    for i in range(N):
        nb = sorted(((i + d) % N) for d in (-3, -2, -1, 1, 2, 3))
        assert list(col[rp[i]:rp[i + 1]]) == nb


def test_ws_csr_seeded():
    a = ws_csr(3000, 8, 0.2, seed=11)
    b = ws_csr(3000, 8, 0.2, seed=11)
    c = ws_csr(3000, 8, 0.2, seed=12)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert not np.array_equal(a[1], c[1])


def test_ws_networkx_seeded():
    rp, col = ws_csr_networkx(400, 8, 0.1, seed=5)
    _check_csr(rp, col, 400, 8)
    rp2, col2 = ws_csr_networkx(400, 8, 0.1, seed=5)
    assert np.array_equal(col, col2)


def test_rewired_fraction():
    N, k, p = 20000, 10, 0.1
    rp, col = ws_csr(N, k, p, seed=1)
    rows = np.repeat(np.arange(N), np.diff(rp))
    dist = np.abs(rows - col)
    dist = np.minimum(dist, N - dist)
    far = np.mean(dist > k // 2)
    # each rewired lattice edge gives two far directed entries
    assert abs(far - p) < 0.01


def test_init_state_distributions():
    rp, _ = ws_csr(1000, 20, 0.1, seed=0)
    st = init_state(rp, 50, seed=0)
    assert st["delays"].dtype == np.uint8
    assert st["delays"].min() >= 1 and st["delays"].max() <= 50
    assert set(np.unique(st["delays"])) == set(range(1, 51))
    assert st["theta"].dtype == np.float32
    assert np.all(st["theta"] >= 0) and np.all(st["theta"] <= np.float32(2 * np.pi))
    assert np.array_equal(st["theta"], st["theta_hat"])
    assert np.all((st["weights"] >= 0) & (st["weights"] < 1))
    assert abs(float(st["omega"].mean())) < 0.15 and abs(float(st["omega"].std()) - 1) < 0.1


def test_config_small_shape():
    net = config_small(0)
    assert net.N == 1000 and net.E == 20000 and net.max_delay == 50


def test_config_batch_small():
    nets, params = config_batch(num=6, seed=0, n_lo=100, n_hi=400)
    assert len(nets) == 6 and len(params) == 6
    assert params[0]["g"] == 0.0 and params[-1]["g"] == 4.0
    assert all(p["gain_controller"] == 0 for p in params)
    for n in nets:
        assert 100 <= n.N <= 400
        assert n.max_delay == 50
        assert n.delays.max() <= 50
