"""ctypes driver of the reference engine built by ``oracle/Makefile``.

TEST INFRASTRUCTURE ONLY (tests/, and the reference arm of bench.py).  Runs
the reference's own ``leviathan_init`` / ``leviathan_step`` / ... C ABI
(leviathan_kernel.cu:270-497 of the reference) on the GPU and reads its
internal state through ``ref_shim_get_state``.  Needs a CUDA device.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIBS = {
    "sm100a": os.path.join(REF_DIR, "libleviathan_ref.so"),
    "stock": os.path.join(REF_DIR, "libleviathan_ref_stock.so"),
}
# Where the reference sources lie (same variable as oracle/Makefile's REF).
REFERENCE_ROOT = os.environ.get("LEVIATHAN_REF", "/root/reference")
REFERENCE_SRC = os.path.join(REFERENCE_ROOT, "src", "cuda", "leviathan_kernel.cu")

_P = C.c_void_p
_cache: dict = {}


def build_if_possible() -> bool:
    """Run oracle/Makefile when the reference sources are present (this
    machine only; the GPU machine uses the prebuilt files)."""
    if not os.path.exists(REFERENCE_SRC):
        return all(os.path.exists(p) for p in LIBS.values())
    proc = subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_ROOT}"],
                          capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("reference build failed:\n" + proc.stdout + proc.stderr)
    return True


def available(flavor: str = "sm100a") -> bool:
    return os.path.exists(LIBS[flavor])


def load(flavor: str = "sm100a") -> C.CDLL:
    if flavor in _cache:
        return _cache[flavor]
    path = LIBS[flavor]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing; run `make -C oracle`")
    lib = C.CDLL(path)
    lib.leviathan_init.restype = _P
    lib.leviathan_init.argtypes = [C.c_int, C.c_int] + [_P] * 7
    lib.leviathan_step.restype = C.c_float
    lib.leviathan_step.argtypes = [_P, C.c_float]
    lib.leviathan_get_theta.argtypes = [_P, _P]
    lib.leviathan_set_theta.argtypes = [_P, _P]
    lib.leviathan_free.argtypes = [_P]
    lib.leviathan_set_gain.argtypes = [_P, C.c_float]
    lib.leviathan_get_gain.restype = C.c_float
    lib.leviathan_get_gain.argtypes = [_P]
    lib.leviathan_set_gain_controller.argtypes = [_P, C.c_bool]
    lib.leviathan_get_vram_usage.restype = C.c_size_t
    lib.leviathan_get_vram_usage.argtypes = [_P]
    lib.leviathan_reset_weights.argtypes = [_P, _P]
    lib.ref_shim_get_state.restype = C.c_int
    lib.ref_shim_get_state.argtypes = [_P] * 6 + [_P, _P]
    lib.ref_shim_stream.restype = _P
    lib.ref_shim_stream.argtypes = [_P]
    _cache[flavor] = lib
    return lib


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class RefEngine:
    """The reference engine (one network) driven through its C ABI."""

    def __init__(self, N, max_delay, row_ptr, col_idx, delays, weights, theta,
                 theta_hat, omega, flavor="sm100a"):
        self.lib = load(flavor)
        self.N = int(N)
        self.max_delay = int(max_delay)
        self._keep = [np.ascontiguousarray(row_ptr, np.int32),
                      np.ascontiguousarray(col_idx, np.int32),
                      np.ascontiguousarray(delays, np.uint8),
                      np.ascontiguousarray(weights, np.float32),
                      np.ascontiguousarray(theta, np.float32),
                      np.ascontiguousarray(theta_hat, np.float32),
                      np.ascontiguousarray(omega, np.float32)]
        self.E = int(self._keep[0][-1])
        self.h = self.lib.leviathan_init(self.N, self.max_delay,
                                         *[_ptr(a) for a in self._keep])
        if not self.h:
            raise RuntimeError("leviathan_init returned NULL")

    def step(self, dt):
        return float(self.lib.leviathan_step(self.h, C.c_float(dt)))

    def run(self, dt, n):
        return np.array([self.step(dt) for _ in range(int(n))], dtype=np.float32)

    def get_theta(self):
        out = np.empty(self.N, np.float32)
        self.lib.leviathan_get_theta(self.h, _ptr(out))
        return out

    def set_theta(self, theta):
        t = np.ascontiguousarray(theta, np.float32)
        self.lib.leviathan_set_theta(self.h, _ptr(t))

    def set_gain(self, g):
        self.lib.leviathan_set_gain(self.h, C.c_float(g))

    def get_gain(self):
        return float(self.lib.leviathan_get_gain(self.h))

    def set_gain_controller(self, enabled):
        self.lib.leviathan_set_gain_controller(self.h, bool(enabled))

    def reset_weights(self, w):
        a = np.ascontiguousarray(w, np.float32)
        self.lib.leviathan_reset_weights(self.h, _ptr(a))

    def get_vram_usage(self):
        return int(self.lib.leviathan_get_vram_usage(self.h))

    def state(self):
        bs = self.max_delay + 1
        th = np.empty(self.N, np.float32)
        thh = np.empty(self.N, np.float32)
        wh = np.empty(self.N, np.float32)
        w = np.empty(max(self.E, 1), np.float32)
        ring = np.empty((self.N, bs), np.float32)
        bi = C.c_int()
        g = C.c_float()
        rc = self.lib.ref_shim_get_state(self.h, _ptr(th), _ptr(thh), _ptr(wh),
                                         _ptr(w), _ptr(ring), C.byref(bi), C.byref(g))
        if rc != 0:
            raise RuntimeError("ref_shim_get_state failed")
        return dict(theta=th, theta_hat=thh, omega_hat=wh, weights=w[: self.E],
                    ring=ring, buf_idx=bi.value, g=g.value)

    @property
    def stream(self):
        return self.lib.ref_shim_stream(self.h)

    def close(self):
        if self.h:
            self.lib.leviathan_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
