"""``LeviathanObservatory``: the reference's high-level host API
(python/leviathan_h100.py:19-219) on the B200 engine.

Same constructor, methods and return values.  Differences, all deliberate:

* the graph and the initial state are seeded (the reference seeds NumPy's
  global generator but calls ``nx.watts_strogatz_graph`` without ``seed=``,
  python/leviathan_h100.py:31-34, so its topology changes from run to run);
* a prebuilt :class:`~leviathan_v1_b200.graphs.Network` can be passed instead
  of (N, k, max_delay, seed) to run a benchmark configuration;
* ``run_baseline`` and ``run_with_stimulus`` advance the engine in step
  blocks (one CUDA-graph replay per block) instead of one host round trip per
  step; they record the same r(t) for every step and print at the same
  intervals.
"""

from __future__ import annotations

import time

import numpy as np

from .engine import LeviathanEngine
from .graphs import Network, init_state, ws_csr_networkx


class LeviathanObservatory:
    """Delayed Kuramoto network with adaptive coupling on one B200."""

    def __init__(self, N=100000, k=20, max_delay=50, seed=42, *, p=0.2,
                 network: Network | None = None, params: dict | None = None,
                 math_mode="reference", verbose=True):
        self.verbose = verbose
        self.dt = 0.05
        if network is None:
            self.N, self.k, self.max_delay = int(N), int(k), int(max_delay)
            self._log(f"[Observatory] Constructing Watts-Strogatz: N={N}, k={k}, p={p}")
            row_ptr, col_idx = ws_csr_networkx(self.N, self.k, p, seed)
            # distributions of python/leviathan_h100.py:51-55
            rng = np.random.default_rng(seed)
            E = int(row_ptr[-1])
            delays = rng.integers(1, max(self.max_delay, 2), E, dtype=np.uint8)
            weights = rng.uniform(0.01, 0.1, E).astype(np.float32)
            theta = rng.uniform(0, 2 * np.pi, self.N).astype(np.float32)
            omega = rng.normal(1.0, 0.1, self.N).astype(np.float32)
            network = Network(self.N, self.max_delay, row_ptr, col_idx, delays,
                              weights, theta, theta.copy(), omega,
                              meta=dict(k=k, p=p, seed=seed))
        else:
            self.N, self.max_delay = network.N, network.max_delay
            self.k = network.meta.get("k", round(network.E / max(network.N, 1)))
        self.network = network
        self.row_ptr = network.row_ptr
        self.col_idx = network.col_idx
        self.nnz = network.E
        self.delays = network.delays
        self.weights = network.weights
        self.theta = network.theta
        self.theta_hat = network.theta_hat
        self.omega = network.omega
        self._log(f"[Observatory] Topology: {self.nnz} edges "
                  f"({self.nnz / max(self.N * max(self.k, 1), 1):.2%} fill)")
        self._log("[Observatory] Initializing B200 CUDA engine...")
        self.engine = LeviathanEngine(*network.engine_args(), params=params,
                                      math_mode=math_mode)
        self._r_capacity = 100000
        self._r_buffer = np.empty(self._r_capacity, dtype=np.float32)
        self.step_count = 0
        self._log("[Observatory] Ready for simulation.\n")

    def _log(self, msg):
        if self.verbose:
            print(msg)

    # -- r history (python/leviathan_h100.py:71-93) -------------------------
    @property
    def r_history(self):
        return self._r_buffer[: self.step_count]

    def _record(self, rs: np.ndarray):
        need = self.step_count + rs.size
        if need > self._r_capacity:
            while self._r_capacity < need:
                self._r_capacity *= 2
            buf = np.empty(self._r_capacity, dtype=np.float32)
            buf[: self.step_count] = self._r_buffer[: self.step_count]
            self._r_buffer = buf
        self._r_buffer[self.step_count: need] = rs
        self.step_count = need

    def step(self):
        """One physics step; returns r."""
        r = self.engine.step(self.dt)
        self._record(np.array([r], dtype=np.float32))
        return r

    def step_n(self, n):
        """``n`` steps in one engine call; returns r[n]."""
        rs = self.engine.step_n(self.dt, n)
        self._record(rs)
        return rs

    # -- controls (python/leviathan_h100.py:95-110) --------------------------
    def set_gain(self, g):
        self.engine.set_gain(g)

    def get_gain(self):
        return self.engine.get_gain()

    def set_gain_controller(self, enabled):
        self.engine.set_gain_controller(enabled)

    def get_vram_usage(self):
        return self.engine.get_vram_usage()

    def reset_weights(self, weights=None):
        if weights is None:
            weights = self.weights
        self.engine.reset_weights(weights)

    def get_vram_report(self):
        """Device-memory report with the layout of python/leviathan_h100.py:
        112-138 (a title line, one line per part, the measured total).  The
        parts are this engine's own buffers: the slot-major delay ring of
        max_delay+2 slots over N rounded up to 32, the four node arrays, the
        per-tile partial sums, and the SELL-32 edge streams with everything
        else as the remainder of the measured total."""
        total = self.get_vram_usage()
        ring = (self.max_delay + 2) * (-(-self.N // 32) * 32) * 4
        nodes = 4 * 4 * self.N
        partials = 8 * -(-self.N // 256)
        parts = [("Delay ring", ring), ("Node state", nodes),
                 ("Tile partials", partials),
                 ("Edges + rest", max(total - ring - nodes - partials, 0))]
        mib = float(1 << 20)
        rule = "-" * 40
        body = "".join(f"{name:20s} : {nbytes / mib:8.2f} MB\n" for name, nbytes in parts)
        return (f"VRAM Usage Report (N={self.N}, E={self.nnz})\n{rule}\n{body}{rule}\n"
                f"{'TOTAL (Measured)':20s} : {total / mib:8.2f} MB\n")

    # -- runs (python/leviathan_h100.py:140-196) -----------------------------
    def run_baseline(self, num_steps=500, log_interval=100):
        """Warm up to metastable criticality; returns r_history."""
        self._log(f"[Observatory] Baseline run: {num_steps} steps")
        start = time.time()
        done = 0
        while done < num_steps:
            n = min(log_interval - (done % log_interval), num_steps - done)
            rs = self.step_n(n)
            done += n
            if done % log_interval == 0:
                fps = done / max(time.time() - start, 1e-12)
                self._log(f"  Step {done:5d}: r={rs[-1]:.4f} ({fps:.1f} FPS)")
        elapsed = time.time() - start
        self._log(f"[Observatory] Complete in {elapsed:.2f}s "
                  f"(avg {num_steps / max(elapsed, 1e-12):.1f} FPS)\n")
        return self.r_history

    def run_with_stimulus(self, num_steps=200, stimulus_start=100,
                          stimulus_nodes=None, stimulus_strength=2.0):
        """External phase kick (TMS-style), python/leviathan_h100.py:157-196.

        Same trajectory as the reference's loop: steps 0 .. stimulus_start
        run, then ``stimulus_strength`` is added to the phase of every listed
        node (a node listed twice is kicked twice), all phases are taken modulo
        2 pi in float32 and uploaded with ``set_phase_snapshot`` (which refills
        the delay ring), and the remaining steps run.  Steps advance in blocks
        (one engine call each) that end at the kick and at every 50th step,
        where the progress line is printed.  Returns r of the last
        ``num_steps`` steps.
        """
        nodes = np.arange(10) if stimulus_nodes is None else np.asarray(stimulus_nodes)
        self._log(f"[Observatory] Stimulus run: {num_steps} steps, start={stimulus_start}")
        self._log(f"[Observatory] Target nodes: {list(nodes[:5])}... (total {nodes.size})")
        self._log(f"[Observatory] Strength: {stimulus_strength}\n")
        kick_after = stimulus_start + 1  # the kick follows step index stimulus_start
        report_every = 50
        t0 = time.time()
        done = 0
        while done < num_steps:
            stops = [num_steps, (done // report_every + 1) * report_every]
            if done < kick_after:
                stops.append(kick_after)
            end = min(stops)
            rs = self.step_n(end - done)
            done = end
            if done == kick_after:
                phases = self.get_phase_snapshot()
                np.add.at(phases, nodes, np.float32(stimulus_strength))
                self.set_phase_snapshot(np.remainder(phases, 2 * np.pi))
                self._log(f"  [STIMULUS] Applied phase kick to {nodes.size} nodes")
            if done % report_every == 0:
                label = "ACTIVE" if done > stimulus_start else "baseline"
                rate = done / max(time.time() - t0, 1e-12)
                self._log(f"  Step {done:3d} [{label}]: r={rs[-1]:.4f} ({rate:.1f} FPS)")
        self._log(f"[Observatory] Complete in {time.time() - t0:.2f}s\n")
        return self.r_history[-num_steps:]

    # -- snapshots (python/leviathan_h100.py:198-219) ------------------------
    def get_phase_snapshot(self):
        return self.engine.get_theta()

    def set_phase_snapshot(self, theta):
        if theta.dtype != np.float32:
            theta = theta.astype(np.float32)
        self.engine.set_theta(theta)

    def statistics(self):
        r_arr = np.array(self.r_history)
        return {
            "final_r": r_arr[-1],
            "mean_r": np.mean(r_arr),
            "max_r": np.max(r_arr),
            "min_r": np.min(r_arr),
            "std_r": np.std(r_arr),
            "steps": len(r_arr),
        }

    def close(self):
        self.engine.close()
