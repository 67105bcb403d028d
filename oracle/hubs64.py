"""CPU restatement of the reference's hub-phase transition counting.

TEST INFRASTRUCTURE ONLY: the checker of ``leviathan_v1_b200.hubs`` and of
the hub observation fused into the engine's step; only ``tests/`` import it.

binarize_and_accumulate_kernel (src/cuda/leviathan_phi_kernel.cu:60-92):
bit i of the state is set when hub i's phase, fmodf'ed by 6.2831853f (plus
6.2831853f if negative), exceeds 3.1415926f -- float32 arithmetic, so the
same constants and np.fmod on float32 (fmod is exact) reproduce it bit for
bit; a NaN phase compares false and gives bit 0.  Each observation counts
the transition from the previous state (none before the first) in an int64
[S][S] matrix and the row totals, and phi_get_transition_count
(:347-349) counts observations.  The reference Python driver's own
binarisation (python/leviathan_iit_integration.py:79-95, ``hub_phases >
np.pi`` on float32 phases, compared in float32 by NumPy >= 2) agrees with it
on the engine's phases, which lie in [0, 2pi), except at the single phase
float32(pi) = 3.14159274, which exceeds 3.1415926f but not float32(pi).
"""

from __future__ import annotations

import numpy as np

TWO_PI_F = np.float32(6.2831853)
PI_F = np.float32(3.1415926)


def hub_state(theta, hubs) -> int:
    phase = np.asarray(theta, np.float32)[np.asarray(hubs)]
    with np.errstate(invalid="ignore"):
        phase = np.fmod(phase, TWO_PI_F)
        phase = np.where(phase < 0, phase + TWO_PI_F, phase).astype(np.float32)
        bits = phase > PI_F
    return int(np.sum(bits.astype(np.int64) << np.arange(len(bits), dtype=np.int64)))


class HubCounter:
    def __init__(self, hubs):
        self.hubs = np.asarray(hubs, np.int64)
        self.S = 1 << len(self.hubs)
        self.counts = np.zeros((self.S, self.S), np.int64)
        self.totals = np.zeros(self.S, np.int64)
        self.prev = -1
        self.observed = 0

    def observe(self, theta) -> int:
        s = hub_state(theta, self.hubs)
        if 0 <= self.prev < self.S:
            self.counts[self.prev, s] += 1
            self.totals[self.prev] += 1
        self.prev = s
        self.observed += 1
        return s
