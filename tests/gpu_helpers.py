"""Helpers shared by the GPU tests."""
from __future__ import annotations

import numpy as np


def config(**kw):
    """A Solver.configure dict with the main.js:9-36 keys."""
    cfg = {"beta": 0.0, "drag": 0.0, "viscosity": 0.0, "hyperP": 4, "forceAmp": 0.0, "forceK": 20.0,
           "forceWidth": 2.0, "cfl": 0.5, "dtMin": 1e-6, "dtMax": 1.0, "dyeFade": 1.0}
    cfg.update(kw)
    return cfg


def rate_for(nu_h, n, p):
    """The viscosity RATE that configure() maps to nu_h (solver.js:311)."""
    return nu_h * (n / 3.0) ** (2 * p)


def set_fixed_dt(solver, dt):
    solver.setBuffer("dt", np.array([dt, 0.0, 0.0, 0.0], np.float32))


def load_state(solver, w, phase=0):
    solver.phase = phase
    solver.setBuffer(f"state{phase}", np.asarray(w).astype(np.complex64))


def current_state(solver):
    return solver.getBuffer(f"state{solver.phase}")
