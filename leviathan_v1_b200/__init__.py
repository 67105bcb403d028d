"""LEVIATHAN core engine step on NVIDIA B200 (sm_100a).

Public surface:

* :class:`LeviathanEngine` -- drop-in for the reference's pybind11 class
  ``leviathan_cuda.LeviathanEngine`` (one network);
* :class:`LeviathanObservatory` -- the reference's host API
  (python/leviathan_h100.py) on this engine;
* :class:`BatchEngine` -- many independent networks per launch;
* :class:`HubTransitions` -- hub-phase transition counts for the
  integrated-information front-end, fed by the engine's own steps;
* :mod:`.graphs` -- seeded topologies and initial states.

The compute path is the CUDA library ``lib/libleviathan_b200.so`` (C ABI in
``include/leviathan_b200.h``); there is no CPU fallback.
"""

from .engine import BatchEngine, LeviathanEngine  # noqa: F401
from .hubs import HubTransitions  # noqa: F401
from .observatory import LeviathanObservatory  # noqa: F401

__all__ = ["LeviathanEngine", "LeviathanObservatory", "BatchEngine", "HubTransitions"]
