"""FP64 NumPy transcription of the LEVIATHAN core engine step.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py``
import it.  The product path (``leviathan_v1_b200``) never does.

It follows the reference kernels line by line (leviathan_kernel.cu in
src/cuda/ of the reference), not docs/MODEL.md where the two differ:

* prep_kernel :93-111 -- eps from the pre-step theta and theta_hat; then
  theta_hat += dt*omega_hat; omega_hat += kappa_w*dt*eps (MODEL.md does not
  state the predictor update);
* csr_physics_kernel :114-167 -- ring slot (buf_idx - d + bs) % bs; the
  coupling sum uses the weight *before* its update; NaN guard to w_min, clamp;
* integrate_and_reduce_kernel :170-234 -- the gain g of the previous
  controller update; wrap to [0, 2pi); NaN guard to 0; ring slot
  (buf_idx + 1) % bs receives the new phase;
* final_reduce_r_kernel :237-264 -- r = |sum exp(i theta)| / N;
* host controller :431-435 -- g += dt*(beta*(r0 - r) - mu*(g - 1.5)), then
  clamp to [g_min, g_max] (g_rest = 1.5 and mu = 0.01 are literals there);
* leviathan_set_theta :445-453 -- theta upload refills every ring slot.

Parity pin: the reference engine itself (leviathan_kernel.cu built from the
unmodified reference sources for sm_100a by ``oracle/Makefile``) was run on a
B200 over seeded fixtures; its outputs are the golden vectors in
``tests/golden/`` (made by ``tests/golden/make_golden.py``) and
``tests/test_oracle.py`` checks this transcription against them.  The
reference has no tests or fixtures of its own.

An optional additive input drive ``drive[i]`` (added to d theta_i / dt) is
supported for the reservoir extension; it is zero for the reference model.
"""

from __future__ import annotations

import numpy as np

TWO_PI = 2.0 * np.pi

DEFAULT_PARAMS = dict(
    # leviathan_kernel.cu:282-296 and the literal g_rest at :433
    eta=0.01, lam=0.001, gamma=0.05, alpha_eps=0.1, kappa_w=0.01,
    w_min=0.0, w_max=2.0, g=1.5, r0=0.5, beta=0.01, mu=0.01, g_rest=1.5,
    g_min=0.1, g_max=5.0, gain_controller=1,
)


class OracleEngine:
    """Reference engine semantics on the CPU, in ``dtype`` (float64 default).

    State layout follows the reference handle (leviathan_kernel.cu:27-72):
    node-major ring ``ring[N, max_delay+1]`` and the slot index ``buf_idx``.
    """

    def __init__(self, N, max_delay, row_ptr, col_idx, delays, weights,
                 theta, theta_hat, omega, params=None, dtype=np.float64):
        self.dtype = np.dtype(dtype)
        f = lambda a: np.array(a, dtype=self.dtype)
        self.N = int(N)
        self.max_delay = int(max_delay)
        self.bs = self.max_delay + 1                       # :277
        self.row_ptr = np.asarray(row_ptr, dtype=np.int64)
        self.col = np.asarray(col_idx, dtype=np.int64)
        self.delays = np.asarray(delays, dtype=np.int64)
        self.E = int(self.row_ptr[-1])                     # :278
        self.row = np.repeat(np.arange(self.N, dtype=np.int64),
                             np.diff(self.row_ptr))
        self.w = f(weights)
        self.theta = f(theta)
        self.theta_hat = f(theta_hat)
        self.omega = f(omega)
        self.omega_hat = f(omega)                          # :350
        self.ring = np.repeat(self.theta[:, None], self.bs, axis=1)  # :79-90
        self.buf_idx = 0
        p = dict(DEFAULT_PARAMS)
        if params:
            p.update(params)
        self.p = p
        self.g = self.dtype.type(p["g"])
        self.ctrl = bool(p["gain_controller"])
        self.t = 0
        self.last_r = None

    # -- helpers ------------------------------------------------------------
    def _wrap_pm_pi(self, x):
        return x - np.floor(x / TWO_PI + 0.5) * TWO_PI     # :105, :146

    def order_parameter(self, theta=None):
        th = self.theta if theta is None else theta
        c = np.cos(th).sum(dtype=np.float64)
        s = np.sin(th).sum(dtype=np.float64)
        return float(np.sqrt(c * c + s * s) / self.N)      # :262

    def ring_slots(self, d):
        return (self.buf_idx - np.asarray(d) + self.bs) % self.bs  # :142

    # -- one step (leviathan_step, :391-438) ----------------------------------
    def step(self, dt, drive=None):
        with np.errstate(invalid="ignore", over="ignore"):
            return self._step(dt, drive)

    def _step(self, dt, drive):
        p = self.p
        T = self.dtype.type
        dt = T(dt)
        # prep_kernel :100-110
        diff = self._wrap_pm_pi(self.theta - self.theta_hat)
        eps = np.sin(diff)
        self.theta_hat = self.theta_hat + dt * self.omega_hat
        self.omega_hat = self.omega_hat + T(p["kappa_w"]) * dt * eps
        # csr_physics_kernel :126-165
        idx = self.ring_slots(self.delays)
        delayed = self.ring[self.col, idx]
        d = self._wrap_pm_pi(delayed - self.theta[self.row])
        sin_d = np.sin(d)
        cos_d = np.cos(d)
        w = self.w
        S = np.bincount(self.row, weights=w * sin_d, minlength=self.N).astype(self.dtype)
        my_eps = np.abs(eps)[self.row]
        dw = dt * (T(p["eta"]) * cos_d * (T(1) - T(p["gamma"]) * my_eps) - T(p["lam"]) * w)
        w = w + dw
        w = np.where(np.isfinite(w), w, T(p["w_min"]))
        self.w = np.clip(w, T(p["w_min"]), T(p["w_max"])).astype(self.dtype)
        # integrate_and_reduce_kernel :183-192
        rate = self.omega + self.g * S - T(p["alpha_eps"]) * eps
        if drive is not None:
            rate = rate + np.asarray(drive, dtype=self.dtype)
        x = self.theta + dt * rate
        x = x - np.floor(x / TWO_PI) * TWO_PI
        x = np.where(np.isfinite(x), x, T(0))
        self.theta = x.astype(self.dtype)
        nxt = (self.buf_idx + 1) % self.bs                 # :406
        self.ring[:, nxt] = self.theta                     # :192
        self.buf_idx = nxt
        # r (:195-262) and host controller (:431-435)
        r = self.order_parameter()
        if self.ctrl:
            g = self.g + dt * (T(p["beta"]) * (T(p["r0"]) - T(r))
                               - T(p["mu"]) * (self.g - T(p["g_rest"])))
            self.g = T(min(max(g, T(p["g_min"])), T(p["g_max"])))
        self.t += 1
        self.last_r = r
        return r

    def run(self, dt, n):
        return np.array([self.step(dt) for _ in range(int(n))], dtype=np.float64)

    # -- state access (leviathan_kernel.cu:440-497) -----------------------------
    def get_theta(self):
        return self.theta.copy()

    def set_theta(self, theta):
        self.theta = np.array(theta, dtype=self.dtype)
        self.ring[:, :] = self.theta[:, None]              # :445-453

    def set_gain(self, g):
        self.g = self.dtype.type(g)

    def get_gain(self):
        return float(self.g)

    def set_gain_controller(self, enabled):
        self.ctrl = bool(enabled)

    def reset_weights(self, w):
        self.w = np.array(w, dtype=self.dtype)


def circular_distance(a, b):
    """|wrap(a - b)| in [0, pi]."""
    d = np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64)
    d = d - np.floor(d / TWO_PI + 0.5) * TWO_PI
    return np.abs(d)


def ring_slot_sequence(max_delay, steps, start=0):
    """buf_idx after each of ``steps`` steps (leviathan_kernel.cu:406,415)."""
    bs = max_delay + 1
    return (start + np.arange(1, steps + 1)) % bs


def edge_slots(buf_idx, delays, max_delay):
    """Ring slot read by each edge at ``buf_idx`` (leviathan_kernel.cu:142)."""
    bs = max_delay + 1
    return (int(buf_idx) - np.asarray(delays, dtype=np.int64) + bs) % bs
