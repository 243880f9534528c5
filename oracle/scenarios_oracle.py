"""CPU restatement of the reference's scenario builders (src/scenarios.js) -- TEST
INFRASTRUCTURE ONLY: the checker for the device-built scenario fields, never part
of the product path.

PARITY UNPINNED: scenarios.js is browser JavaScript with no test, fixture or
runnable copy in the reference (Node is not available here); this follows its
formulas line by line in FP64 and rounds to float32 like its Float32Array.
"""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 2.0 * math.pi


def _grid(n):                                    # scenarios.js:3-13
    h = TWO_PI / n
    idx = np.arange(n, dtype=np.float64)
    x = (idx * h)[None, :]
    y = (idx * h)[:, None]
    return x, y


def _wrap_delta(a, b):                           # scenarios.js:20-28
    d = a - b
    d = np.where(d > math.pi, d - TWO_PI, d)
    return np.where(d < -math.pi, d + TWO_PI, d)


def _blobs(n, blobs):                            # scenarios.js:30-44
    x, y = _grid(n)
    acc = np.zeros((n, n))
    for bx, by, a, amp in blobs:
        dx = _wrap_delta(x, bx)
        dy = _wrap_delta(y, by)
        r2 = dx * dx + dy * dy
        s2 = a * a
        acc = acc + np.where(r2 < 25 * s2, amp * np.exp(-r2 / s2), 0.0)
    return acc


def _ring(n, count, radius, a, amp, jitter):     # scenarios.js:46-56
    mode = max(2, count // 2)
    blobs = []
    for j in range(count):
        th = TWO_PI * j / count
        r = radius * (1 + jitter * math.cos(TWO_PI * mode * j / count))
        blobs.append((math.pi + r * math.cos(th), math.pi + r * math.sin(th), a, amp))
    return _blobs(n, blobs)


def build(name, n, cfg=None):
    cfg = cfg or {}
    x, y = _grid(n)
    if name == "shear layer":                    # scenarios.js:70-79
        delta = max(TWO_PI / 30, 6 * TWO_PI / n)
        eps = 0.05
        lower = y <= math.pi
        z = np.where(lower, (y - math.pi / 2) / delta, (1.5 * math.pi - y) / delta)
        dudy = np.where(lower, 1.0, -1.0) * (1.0 / np.cosh(z) ** 2) / delta
        f = eps * np.cos(x) - dudy
    elif name == "taylor-green":                 # scenarios.js:94-97
        f = 6 * np.cos(2 * x) * np.cos(2 * y)
    elif name == "dipole":                       # scenarios.js:112-122
        gamma, a, d = 12.0, 0.3, 0.9
        amp = gamma / (math.pi * a * a)
        cx = math.pi * 0.6
        f = _blobs(n, [(cx, math.pi - d / 2, a, amp), (cx, math.pi + d / 2, a, -amp)])
    elif name == "merger":                       # scenarios.js:136-143
        a, d = 0.22, float(cfg.get("mergerSep", 0.7))
        f = _blobs(n, [(math.pi - d / 2, math.pi, a, 30.0), (math.pi + d / 2, math.pi, a, 30.0)])
    elif name == "polygon":                      # scenarios.js:157-159
        f = _ring(n, int(math.floor(float(cfg.get("polygonN", 6)) + 0.5)), 1.25, 0.19, 34.0, 0.02)
    else:
        raise ValueError(name)
    return np.broadcast_to(f, (n, n)).astype(np.float32)
