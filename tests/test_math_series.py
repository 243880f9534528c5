"""Truncation bounds of the series the stage kernels use for the integrating factor
(expm1_series, sincos_series in csrc/s2d_device.cuh), evaluated in float64 with the
same terms: the series part must stay far below FP32 rounding (6e-8) over its whole
domain; the device results themselves are checked against the FP64 oracle by the GPU
parity tests (fused step, Taylor-Green decay, inviscid invariants, ensembles)."""
import math

import numpy as np


def expm1_series(x):
    p = 1.0 / 5040.0
    for c in (1 / 720, 1 / 120, 1 / 24, 1 / 6, 0.5, 1.0):
        p = p * x + c
    return p * x


def sincos_series(a):
    a2 = a * a
    ps = 1.0 / 362880.0
    for c in (-1 / 5040, 1 / 120, -1 / 6, 1.0):
        ps = ps * a2 + c
    pc = -1.0 / 3628800.0
    for c in (1 / 40320, -1 / 720, 1 / 24, -0.5):
        pc = pc * a2 + c
    return ps * a, pc * a2 + 1.0


def test_expm1_series_bound():
    x = np.concatenate([np.linspace(-0.25, 0.25, 20001), np.geomspace(1e-12, 0.25, 2000),
                        -np.geomspace(1e-12, 0.25, 2000)])
    x = x[np.abs(x) < 0.25]
    rel = np.abs(expm1_series(x) - np.expm1(x)) / np.maximum(np.abs(np.expm1(x)), 1e-300)
    assert rel.max() < 2e-9, rel.max()


def test_sincos_series_bound():
    a = np.concatenate([np.linspace(-math.pi / 4, math.pi / 4, 20001), np.geomspace(1e-12, math.pi / 4, 2000)])
    s, c = sincos_series(a)
    rs = np.abs(s - np.sin(a)) / np.maximum(np.abs(np.sin(a)), 1e-300)
    rc = np.abs(c - np.cos(a))
    assert rs.max() < 3e-9, rs.max()
    assert rc.max() < 3e-9, rc.max()
