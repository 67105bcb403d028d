"""Hub-phase transition counts: the integrated-information front-end.

The reference estimates a transition probability matrix of up to 10 hub
nodes for its integrated-information solver.  After every step the hub phases
are binarised -- bit i set when hub i's phase, taken modulo 6.2831853f into
[0, 2pi), exceeds 3.1415926f -- and the transition from the previous state is
counted (binarize_and_accumulate_kernel, src/cuda/leviathan_phi_kernel.cu:
60-92).  Its Python driver takes a host snapshot of all N phases every step
to do so (python/leviathan_iit_integration.py:244-250).

``HubTransitions`` keeps the counts on the device.  ``attach(engine)`` makes
the engine observe the hubs inside every step's own reduction (no snapshot,
no extra launch); ``accumulate(theta)`` observes one phase array, like the
reference binding's ``GPUPhiWorker.accumulate``
(src/bindings/leviathan_phi_pybind.cpp:37-55).  ``tpm()`` and ``sbn_tpm()``
normalise the counts on the host as normalize_tpm_kernel and
build_sbn_tpm_kernel do (leviathan_phi_kernel.cu:98-136).  The
integrated-information solver itself is not part of this library.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

MAX_HUBS = 10


class HubTransitions:
    def __init__(self, hub_indices):
        idx = np.ascontiguousarray(np.asarray(hub_indices), dtype=np.int32)
        if idx.ndim != 1 or not 1 <= idx.size <= MAX_HUBS:
            raise ValueError(f"1 to {MAX_HUBS} hub indices are required")
        self._lib = _lib.load()
        self.hub_indices = idx
        self.num_hubs = int(idx.size)
        self.num_states = 1 << self.num_hubs
        self._h = C.c_void_p(0)
        check(self._lib.lev_hubs_create(C.byref(self._h), self.num_hubs,
                                        C.c_void_p(idx.ctypes.data)))
        self._engine = None
        self._dev_theta = None

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.lev_hubs_destroy(self._h)
            self._h = C.c_void_p(0)
        self._engine = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        if not self._h.value:
            raise RuntimeError("hub monitor is closed")
        return self._h

    # -- feeding ------------------------------------------------------------
    def attach(self, engine, net: int = 0) -> None:
        """Observe every later step of network ``net`` of ``engine``."""
        check(self._lib.lev_attach_hubs(engine.handle, int(net), self.handle))
        self._engine = engine

    def detach(self) -> None:
        if self._engine is not None:
            check(self._lib.lev_attach_hubs(self._engine.handle, 0, None))
            self._engine = None

    def accumulate(self, theta) -> None:
        """One observation of a phase array: a CUDA tensor (used in place) or
        host data (copied to the device first, as GPUPhiWorker.accumulate
        does)."""
        import torch

        if isinstance(theta, torch.Tensor) and theta.is_cuda:
            t = theta.detach().to(torch.float32).contiguous()
        else:
            t = torch.as_tensor(np.ascontiguousarray(theta, dtype=np.float32)).cuda()
        if t.numel() <= int(self.hub_indices.max()):
            raise ValueError("phase array shorter than the largest hub index")
        self._dev_theta = t  # kept alive until the observation has run
        stream = torch.cuda.current_stream(t.device).cuda_stream
        check(self._lib.lev_hubs_accumulate(self.handle, C.c_void_p(t.data_ptr()),
                                            C.c_void_p(stream)))

    def reset(self) -> None:
        check(self._lib.lev_hubs_reset(self.handle))

    # -- results ------------------------------------------------------------
    def read(self):
        """(counts[S, S] uint64 with rows = previous state, totals[S],
        last state (-1 before any observation), observations)."""
        S = self.num_states
        counts = np.empty((S, S), np.uint64)
        totals = np.empty(S, np.uint64)
        prev = C.c_int32()
        obs = C.c_int64()
        check(self._lib.lev_hubs_read(self.handle, C.c_void_p(counts.ctypes.data),
                                      C.c_void_p(totals.ctypes.data), C.byref(prev),
                                      C.byref(obs)))
        return counts, totals, prev.value, obs.value

    def get_transition_count(self) -> int:
        """Observations so far (phi_get_transition_count)."""
        return self.read()[3]

    def tpm(self) -> np.ndarray:
        """P(state at t+1 | state at t), float32; rows never left are
        uniform (normalize_tpm_kernel, leviathan_phi_kernel.cu:98-115, here
        with IEEE division where the kernel uses the approximate
        __fdividef)."""
        counts, totals, _, _ = self.read()
        S = self.num_states
        out = np.full((S, S), np.float32(1.0) / np.float32(S), np.float32)
        seen = totals > 0
        out[seen] = (counts[seen].astype(np.float32) /
                     totals[seen, None].astype(np.float32))
        return out

    def sbn_tpm(self) -> np.ndarray:
        """P(hub n on at t+1 | state at t), [S, num_hubs] (build_sbn_tpm_kernel,
        leviathan_phi_kernel.cu:121-136)."""
        tpm = self.tpm()
        S, H = self.num_states, self.num_hubs
        bits = ((np.arange(S)[:, None] >> np.arange(H)) & 1).astype(np.float32)
        out = np.zeros((S, H), np.float32)
        for t in range(S):  # float32 sums in the kernel's order over t
            out += tpm[:, t:t + 1] * bits[t]
        return out
