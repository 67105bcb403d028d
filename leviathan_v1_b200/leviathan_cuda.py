"""Module-name alias of the reference binding: ``leviathan_cuda``
(src/bindings/leviathan_pybind11.cpp:82).  Code written against the reference
switches engines by importing ``LeviathanEngine`` from here instead."""

from .engine import LeviathanEngine  # noqa: F401

__all__ = ["LeviathanEngine"]
