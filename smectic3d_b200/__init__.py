"""B200-native (sm_100a) pseudo-spectral Swift-Hohenberg time loop of smectic3D.

The compute path is ``libsmectic_b200.so`` (hand-written CUDA, C-ABI in
include/smectic_b200.h); this package is its host-side mirror.
"""
from .solver import Params, Solver  # noqa: F401
from . import ic  # noqa: F401
from ._lib import ShError, load as load_library  # noqa: F401

__all__ = ["Params", "Solver", "ShError", "load_library", "ic"]
