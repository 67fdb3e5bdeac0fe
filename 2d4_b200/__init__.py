"""B200 engine for the 2D4_sim implicit-step hot path.

The package is named ``2d4_b200``; import it with
``importlib.import_module("2d4_b200")``.  The compute path is libd4core.so
(hand-written sm_100a CUDA behind the C ABI of include/d4core.h).
"""
from . import _lib, dconf
from .ensemble import Ensemble
from .simulation import (CyclicLoadProtocol, Engine, Field, FixedRateProtocol,
                         FixedRateStressProtocolObject, IncreasingCyclicLoadProtocol, Simulation,
                         SimulationData, StressProtocol, StressProtocolObject)

__all__ = ["_lib", "dconf", "Engine", "Ensemble", "Field", "Simulation", "SimulationData", "StressProtocol",
           "StressProtocolObject", "FixedRateProtocol", "FixedRateStressProtocolObject",
           "CyclicLoadProtocol", "IncreasingCyclicLoadProtocol"]
