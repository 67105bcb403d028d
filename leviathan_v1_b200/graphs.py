"""Seeded Watts-Strogatz topologies, CSR conversion and initial states.

The reference builds its topology with ``networkx.watts_strogatz_graph(N, k,
p)`` and converts it with ``nx.to_scipy_sparse_array(G, format="csr")``
(python/leviathan_h100.py:34-45), without a seed (the graph changes from run
to run).  Two generators are provided here, both seeded:

* ``ws_csr_networkx`` calls the same networkx routine with ``seed=`` and the
  same CSR conversion; used for the small configurations;
* ``ws_csr`` is a vectorised NumPy generator of the same model (ring lattice
  of k/2 neighbours per side, each lattice edge (u, u+j) rewired with
  probability p to (u, w), w uniform, no self-loops or multi-edges) that
  produces the canonical CSR (symmetric, int32, columns sorted per row) in
  seconds at N = 10^6.

Initial states follow the distributions of the benchmark configurations
(delays uniform in [1, max_delay], omega ~ Normal(mean, std), theta uniform in
[0, 2pi), theta_hat = theta, weights uniform in [w_lo, w_hi)).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def _edges_to_csr(u: np.ndarray, v: np.ndarray, N: int):
    """Undirected edge list -> symmetric CSR (row_ptr int32, col_idx int32)."""
    rows = np.concatenate([u, v]).astype(np.int64)
    cols = np.concatenate([v, u]).astype(np.int64)
    key = rows * N + cols
    key.sort(kind="stable")
    rows = key // N
    cols = key - rows * N
    counts = np.bincount(rows, minlength=N)
    row_ptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    if row_ptr[-1] >= 2**31:
        raise ValueError("graph too large for int32 CSR")
    return row_ptr.astype(np.int32), cols.astype(np.int32)


def ws_csr(N: int, k: int, p: float, seed: int):
    """Vectorised seeded Watts-Strogatz graph as CSR (row_ptr, col_idx)."""
    if k % 2 or k < 2 or k >= N:
        raise ValueError("k must be even with 2 <= k < N")
    rng = np.random.default_rng(seed)
    half = k // 2
    u = np.repeat(np.arange(N, dtype=np.int64), half)
    v = (u + np.tile(np.arange(1, half + 1, dtype=np.int64), N)) % N
    rewire = rng.random(u.size) < p
    keep_u, keep_v = u[~rewire], v[~rewire]
    lo = np.minimum(keep_u, keep_v)
    hi = np.maximum(keep_u, keep_v)
    existing = np.sort(lo * N + hi)
    pend_u = u[rewire]
    new_u, new_v = [], []
    while pend_u.size:
        w = rng.integers(0, N, pend_u.size, dtype=np.int64)
        key = np.minimum(pend_u, w) * N + np.maximum(pend_u, w)
        ok = w != pend_u
        pos = np.searchsorted(existing, key)
        pos = np.minimum(pos, existing.size - 1) if existing.size else pos
        if existing.size:
            ok &= existing[pos] != key
        # first occurrence wins among candidates drawn in the same round
        _, first = np.unique(key, return_index=True)
        is_first = np.zeros(key.size, dtype=bool)
        is_first[first] = True
        ok &= is_first
        new_u.append(pend_u[ok])
        new_v.append(w[ok])
        existing = np.sort(np.concatenate([existing, key[ok]]))
        pend_u = pend_u[~ok]
    eu = np.concatenate([keep_u] + new_u)
    ev = np.concatenate([keep_v] + new_v)
    return _edges_to_csr(eu, ev, N)


def ws_csr_networkx(N: int, k: int, p: float, seed: int):
    """Seeded ``networkx.watts_strogatz_graph`` + scipy CSR, the calls of
    python/leviathan_h100.py:34-45."""
    import networkx as nx

    G = nx.watts_strogatz_graph(N, k=k, p=p, seed=seed)
    A = nx.to_scipy_sparse_array(G, format="csr")
    return A.indptr.astype(np.int32), A.indices.astype(np.int32)


@dataclass
class Network:
    """One network: topology + initial state, in the engine's dtypes."""

    N: int
    max_delay: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    delays: np.ndarray
    weights: np.ndarray
    theta: np.ndarray
    theta_hat: np.ndarray
    omega: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def E(self) -> int:
        return int(self.row_ptr[-1])

    def as_dict(self) -> dict:
        return dict(N=self.N, max_delay=self.max_delay, row_ptr=self.row_ptr,
                    col_idx=self.col_idx, delays=self.delays,
                    weights=self.weights, theta=self.theta,
                    theta_hat=self.theta_hat, omega=self.omega)

    def engine_args(self):
        """Positional arguments of ``LeviathanEngine(...)`` (the reference
        constructor order, leviathan_pybind11.cpp:86-89)."""
        return (self.N, self.max_delay, self.row_ptr, self.col_idx, self.delays,
                self.weights, self.theta, self.theta_hat, self.omega)

    def save(self, path: str) -> None:
        np.savez_compressed(path, N=self.N, max_delay=self.max_delay,
                            row_ptr=self.row_ptr, col_idx=self.col_idx,
                            delays=self.delays, weights=self.weights,
                            theta=self.theta, theta_hat=self.theta_hat,
                            omega=self.omega)

    @staticmethod
    def load(path: str) -> "Network":
        z = np.load(path)
        return Network(int(z["N"]), int(z["max_delay"]), z["row_ptr"], z["col_idx"],
                       z["delays"], z["weights"], z["theta"], z["theta_hat"],
                       z["omega"])


def init_state(row_ptr: np.ndarray, max_delay: int, seed: int, *,
               delay_lo: int = 1, delay_hi: int | None = None,
               omega_mean: float = 0.0, omega_std: float = 1.0,
               w_lo: float = 0.0, w_hi: float = 1.0) -> dict:
    """Seeded initial state (drawn in a fixed order from one generator)."""
    N = row_ptr.size - 1
    E = int(row_ptr[-1])
    if delay_hi is None:
        delay_hi = max_delay
    rng = np.random.default_rng([seed, 0x1E71A7])
    delays = rng.integers(delay_lo, delay_hi + 1, E, dtype=np.uint8)
    omega = rng.normal(omega_mean, omega_std, N).astype(np.float32)
    theta = rng.uniform(0.0, 2.0 * np.pi, N).astype(np.float32)
    weights = rng.uniform(w_lo, w_hi, E).astype(np.float32)
    return dict(delays=delays, omega=omega, theta=theta, theta_hat=theta.copy(),
                weights=weights)


def make_network(N: int, k: int, p: float, max_delay: int, seed: int, *,
                 generator: str = "numpy", **state_kw) -> Network:
    if generator == "networkx":
        rp, col = ws_csr_networkx(N, k, p, seed)
    else:
        rp, col = ws_csr(N, k, p, seed)
    st = init_state(rp, max_delay, seed, **state_kw)
    return Network(N, max_delay, rp, col, st["delays"], st["weights"], st["theta"],
                   st["theta_hat"], st["omega"],
                   meta=dict(k=k, p=p, seed=seed, generator=generator))


def make_network_gpu(N: int, k: int, p: float, max_delay: int, seed: int, *,
                     delay_lo: int = 1, delay_hi: int | None = None,
                     omega_mean: float = 0.0, omega_std: float = 1.0,
                     w_lo: float = 0.0, w_hi: float = 1.0) -> Network:
    """Seeded Watts-Strogatz network and initial state built on the GPU
    (``lev_gen_ws``): the same random-graph model as ``ws_csr`` with device
    random streams, in milliseconds at N = 10^6."""
    import ctypes as C

    from . import _lib

    lib = _lib.load()
    if delay_hi is None:
        delay_hi = max_delay
    E = N * k
    rp = np.empty(N + 1, np.int32)
    col = np.empty(E, np.int32)
    dl = np.empty(E, np.uint8)
    w = np.empty(E, np.float32)
    th = np.empty(N, np.float32)
    om = np.empty(N, np.float32)
    P = lambda a: C.c_void_p(a.ctypes.data)
    _lib.check(lib.lev_gen_ws(int(N), int(k), float(p), int(seed) & (2**64 - 1),
                              int(delay_lo), int(delay_hi), float(w_lo), float(w_hi),
                              float(omega_mean), float(omega_std), P(rp), P(col), P(dl),
                              P(w), P(th), P(om)))
    return Network(N, max_delay, rp, col, dl, w, th, th.copy(), om,
                   meta=dict(k=k, p=p, seed=seed, generator="gpu"))


# ---------------------------------------------------------------------------
# Benchmark configurations (synthetic, seeded)
# ---------------------------------------------------------------------------
DT = 0.05


def config_small(seed: int = 0) -> Network:
    """Plain engine, small: WS N=1000, k=20, p=0.1 (networkx, seeded);
    delays uniform [1,50]; omega ~ N(0,1); theta ~ U[0,2pi); w ~ U[0,1)."""
    return make_network(1000, 20, 0.1, 50, seed, generator="networkx")


def config_scale(seed: int = 0, N: int = 1_000_000, k: int = 32) -> Network:
    """Plain engine at scale: WS N=10^6, k=32, p=0.1; delays [1,64]."""
    return make_network(N, k, 0.1, 64, seed)


def batch_specs(num: int = 512, seed: int = 0, n_lo: int = 500,
                n_hi: int = 50_000, ks=(8, 16, 20, 32)):
    """Specifications of the batched sweep without building the graphs:
    list of dicts (N, k, seed, K, E).  E = N*k exactly (WS rewiring moves
    edges, it never adds or removes them)."""
    rng = np.random.default_rng([seed, 0xBA7C4])
    specs = []
    for b in range(num):
        N = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        k = int(rng.choice(ks))
        k = min(k, N - 2 - (N % 2))
        K = 4.0 * b / max(num - 1, 1)
        specs.append(dict(index=b, N=N, k=k, seed=seed * 100003 + b, K=K, E=N * k))
    return specs


def build_batch(specs):
    """Networks and parameters (K swept, controller off) of ``specs``."""
    nets = [make_network(s["N"], s["k"], 0.1, 50, s["seed"]) for s in specs]
    params = [dict(g=s["K"], gain_controller=0) for s in specs]
    return nets, params


def config_batch(num: int = 512, seed: int = 0, n_lo: int = 500,
                 n_hi: int = 50_000, ks=(8, 16, 20, 32)):
    """Batched sweep: ``num`` networks, N log-uniform in [n_lo, n_hi], k
    uniform in ``ks``, p=0.1, delays [1,50]; coupling K swept linearly over
    [0, 4] with the controller off.  Returns (networks, params)."""
    return build_batch(batch_specs(num, seed, n_lo, n_hi, ks))


def config_adjoint(seed: int = 0, N: int = 10_000, k: int = 20) -> Network:
    """Adjoint: WS N=10^4, k=20, delays [1,50]."""
    return make_network(N, k, 0.1, 50, seed)


def config_reservoir(seed: int = 0, N: int = 50_000, k: int = 20) -> Network:
    """Differentiable reservoir: WS N=5*10^4, k=20, delays [1,50]."""
    return make_network(N, k, 0.1, 50, seed)
