"""yukawamd_b200: B200 (sm_100a) force-and-integrate engine for the O(N^2)
Yukawa / nucleon pair sums and velocity-Verlet updates of MD 6.2.0.

The compute path is the CUDA library libyukawa_b200.so behind the C-ABI of
include/yukawa_engine.h; this package is its host-side mirror of the
reference's accel(do_measurements) / newton(do_measurements) interface.
"""
from . import abi  # noqa: F401
from ._lib import EngineError, lib  # noqa: F401
from .engine import Batch, Engine  # noqa: F401

__all__ = ["abi", "Batch", "Engine", "EngineError", "lib"]
