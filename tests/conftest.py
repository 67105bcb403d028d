"""Shared fixtures of the test suite.

Markers: ``gpu`` -- needs a CUDA device (B200); everything else runs on CPU.
"""

from __future__ import annotations

import glob
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
for p in (REPO, os.path.join(REPO, "oracle"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def golden_cases():
    return [os.path.splitext(os.path.basename(f))[0] for f in golden_files()]


def load_golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def network_from_golden(z):
    from leviathan_v1_b200.graphs import Network

    return Network(int(z["N"]), int(z["max_delay"]), z["row_ptr"], z["col_idx"],
                   z["delays"], z["weights"], z["theta"], z["theta_hat"], z["omega"])


def record_from_golden(z):
    rec = {"theta": [], "weights": [], "predictor": [], "ring": []}
    for k in z.files:
        if "@" not in k:
            continue
        name, t = k.split("@")
        t = int(t)
        if name == "theta":
            rec["theta"].append(t)
        elif name == "weights":
            rec["weights"].append(t)
        elif name == "theta_hat":
            rec["predictor"].append(t)
        elif name == "ring":
            rec["ring"].append(t)
    return rec


class LevAdapter:
    """B200 engine behind the replay interface of make_golden.replay."""

    def __init__(self, net, math_mode="reference"):
        from leviathan_v1_b200 import LeviathanEngine

        self.e = LeviathanEngine(*net.engine_args(), math_mode=math_mode)

    def step(self, dt):
        return self.e.step(dt)

    def get_theta(self):
        return self.e.get_theta()

    def set_theta(self, t):
        self.e.set_theta(t)

    def set_gain(self, g):
        self.e.set_gain(g)

    def set_gain_controller(self, on):
        self.e.set_gain_controller(on)

    def state(self):
        th_hat, om_hat = self.e.get_predictor()
        ring, bi = self.e.get_ring(0)
        return dict(theta=self.e.get_theta(), theta_hat=th_hat, omega_hat=om_hat,
                    weights=self.e.get_weights(), ring=ring, buf_idx=bi,
                    g=self.e.get_gain())

    def close(self):
        self.e.close()


class OracleAdapter:
    """FP64 oracle behind the replay interface."""

    def __init__(self, net, dtype=np.float64):
        from oracle64 import OracleEngine

        self.o = OracleEngine(*net.engine_args(), dtype=dtype)

    def step(self, dt):
        return self.o.step(dt)

    def get_theta(self):
        return self.o.get_theta().astype(np.float32)

    def set_theta(self, t):
        self.o.set_theta(np.asarray(t, np.float32))

    def set_gain(self, g):
        self.o.set_gain(np.float32(g))

    def set_gain_controller(self, on):
        self.o.set_gain_controller(on)

    def state(self):
        o = self.o
        return dict(theta=o.theta.copy(), theta_hat=o.theta_hat.copy(),
                    omega_hat=o.omega_hat.copy(), weights=o.w.copy(),
                    ring=o.ring.copy(), buf_idx=o.buf_idx, g=float(o.g))

    def close(self):
        pass


@pytest.fixture(scope="session")
def gpu_lib():
    if not has_gpu():
        pytest.skip("no CUDA device")
    from leviathan_v1_b200 import _lib

    return _lib.load()
