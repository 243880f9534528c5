"""Scenario presets of the reference (src/scenarios.js, SCENARIOS) on the device.

``SCENARIOS[name]`` holds the reference's ``config`` block (the physics keys feed
``Solver.configure``; the render keys are kept as data) and the kernel id of its
``build(n, cfg)``.  ``build(solver, name, cfg)`` returns the field the reference's
``build`` would return (n*n float32, row-major), evaluated on the GPU;
``Solver.resetScenario`` seeds from it without the field leaving the device
(main.js:281-283: ``solver.reset({ field: scenario.build(config.resolution, config) })``).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L

_RENDER = {"mode": "vorticity", "vortScale": 0.16, "exposure": 1.3}

SCENARIOS = {
    "shear layer": {"kind": L.S2D_SCENARIO_SHEAR_LAYER, "param": None,            # scenarios.js:58-80
                    "config": {"substeps": 2, "viscosity": 0.5, "hyperP": 4, "beta": 0, "drag": 0,
                               "forceAmp": 0, **_RENDER}},
    "taylor-green": {"kind": L.S2D_SCENARIO_TAYLOR_GREEN, "param": None,         # scenarios.js:82-98
                     "config": {"substeps": 4, "viscosity": 90, "hyperP": 1, "beta": 0, "drag": 0,
                                "forceAmp": 0, **_RENDER}},
    "dipole": {"kind": L.S2D_SCENARIO_DIPOLE, "param": None,                     # scenarios.js:100-123
               "config": {"substeps": 4, "viscosity": 0.3, "hyperP": 4, "beta": 0, "drag": 0,
                          "forceAmp": 0, "mode": "dye over vorticity", "vortScale": 0.022, "exposure": 1.3}},
    "merger": {"kind": L.S2D_SCENARIO_MERGER, "param": "mergerSep",              # scenarios.js:125-144
               "config": {"substeps": 8, "viscosity": 0.3, "hyperP": 4, "beta": 0, "drag": 0,
                          "forceAmp": 0, "mode": "vorticity", "vortScale": 0.032, "exposure": 1.3}},
    "polygon": {"kind": L.S2D_SCENARIO_POLYGON, "param": "polygonN",             # scenarios.js:146-160
                "config": {"substeps": 8, "viscosity": 0.22, "hyperP": 4, "beta": 0, "drag": 0,
                           "forceAmp": 0, "mode": "vorticity", "vortScale": 0.026, "exposure": 1.3}},
}
SCENARIO_NAMES = list(SCENARIOS)
# main.js:29-30 defaults of the two scenario parameters
DEFAULT_PARAMS = {"polygonN": 6, "mergerSep": 0.7}


def _kind_param(name: str, cfg: dict | None):
    if name not in SCENARIOS:
        raise ValueError(f"unknown scenario {name!r}; one of {SCENARIO_NAMES}")
    sc = SCENARIOS[name]
    key = sc["param"]
    param = 0.0 if key is None else float((cfg or {}).get(key, DEFAULT_PARAMS[key]))
    return sc["kind"], param


def build(solver, name: str, cfg: dict | None = None) -> np.ndarray:
    """SCENARIOS[name].build(solver.n, cfg): the physical vorticity field, (n, n) float32."""
    kind, param = _kind_param(name, cfg)
    out = np.empty((solver.n, solver.n), np.float32)
    L.call("s2d_scenario_field", solver._use(), kind, param, out.ctypes.data_as(L.C.POINTER(L.C.c_float)))
    return out


def reset(solver, name: str, cfg: dict | None = None, dyePattern: str = "bands"):
    """reset({field: SCENARIOS[name].build(n, cfg), dyePattern}) with the field built on the device."""
    from .solver import _PATTERNS
    if dyePattern not in _PATTERNS:
        raise ValueError(f"unknown dye pattern {dyePattern!r}")
    kind, param = _kind_param(name, cfg)
    L.call("s2d_reset_scenario", solver._use(), kind, param, _PATTERNS[dyePattern])
