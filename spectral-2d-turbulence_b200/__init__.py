"""B200-native integrating-factor RK3 pseudo-spectral vorticity solver.

Drop-in for the step path of the reference's JavaScript solver API
(``src/gpu/solver.js``, ``src/gpu/fft.js``, ``src/gpu/device.js``): the same
``Solver`` methods over the C ABI of ``libs2d.so`` (``include/s2d.h``), which
runs hand-written sm_100a CUDA.  There is no CPU fallback: without a built
library and a B200 the calls raise.
"""
from ._lib import LIB_PATH, S2DError, lib
from .ensemble import Ensemble
from .pointer import Pointer
from .scenarios import SCENARIO_NAMES, SCENARIOS
from .solver import (MAX_SPLATS, Fft2D, Solver, dealiasMaskTable, digitReverseTable, radixSchedule,
                     supportedGrids, wavenumberTable)

__all__ = [
    "Solver", "Fft2D", "Ensemble", "S2DError", "MAX_SPLATS", "radixSchedule", "supportedGrids",
    "digitReverseTable", "wavenumberTable", "dealiasMaskTable", "lib", "LIB_PATH", "SCENARIOS",
    "SCENARIO_NAMES", "Pointer",
]
