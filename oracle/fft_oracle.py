"""Restatement of the reference FFT model ``reference/fft_ref.py``.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Pinned against the
digit-reversal tables and line transforms that ``reference/fft_ref.py``
produced in the development container (``tests/golden/fft_golden.npz``).
"""
from __future__ import annotations

import numpy as np

TWO_PI = 2.0 * np.pi


def radix_schedule(n: int) -> list[int]:
    """Radix list [4, ..., 4, (2)] for n = 4^a or 2*4^a (fft_ref.py:6-16, fft.js:20-31)."""
    out = []
    m = int(n)
    while m % 4 == 0 and m > 1:
        out.append(4)
        m //= 4
    if m == 2:
        out.append(2)
    elif m != 1:
        raise ValueError(f"grid size {n} must be 4^a or 2 * 4^a")
    return out


def digit_reverse(i: int, radices: list[int]) -> int:
    """Mixed-radix digit reversal taken over the REVERSED radix list (fft_ref.py:19-24)."""
    out = 0
    for r in radices[::-1]:
        out = out * r + (i % r)
        i //= r
    return out


def digit_reverse_table(n: int) -> np.ndarray:
    """Permutation used by the reference's load scatter (fft.wgsl:32-49), as uint32."""
    rad = radix_schedule(n)
    return np.array([digit_reverse(i, rad) for i in range(n)], dtype=np.uint32)


def dit_line(x, inverse=False):
    """In-place radix-4 (+ trailing radix-2) DIT line transform (fft_ref.py:27-69).

    Vectorised over butterflies per stage; same arithmetic order as the model.
    Forward is unscaled with sign -1, inverse has sign +1 and scale 1/n.
    """
    x = np.asarray(x, np.complex128)
    n = x.shape[0]
    rad = radix_schedule(n)
    sgn = 1.0 if inverse else -1.0
    buf = np.empty(n, np.complex128)
    buf[digit_reverse_table(n).astype(np.int64)] = x
    m = 1
    for r in rad:
        bt = np.arange(n // r)
        j = bt % m
        base = (bt // m) * r * m + j
        ang = sgn * TWO_PI * j / (r * m)
        if r == 4:
            a0 = buf[base]
            a1 = buf[base + m] * np.exp(1j * ang)
            a2 = buf[base + 2 * m] * np.exp(2j * ang)
            a3 = buf[base + 3 * m] * np.exp(3j * ang)
            b0, b1, b2, b3 = a0 + a2, a0 - a2, a1 + a3, 1j * sgn * (a1 - a3)
            buf[base], buf[base + m] = b0 + b2, b1 + b3
            buf[base + 2 * m], buf[base + 3 * m] = b0 - b2, b1 - b3
        else:
            a0 = buf[base]
            a1 = buf[base + m] * np.exp(1j * ang)
            buf[base], buf[base + m] = a0 + a1, a0 - a1
        m *= r
    if m != n:
        raise AssertionError(f"radix schedule reached m={m} for N={n}")
    return buf / n if inverse else buf


def fft2_model(a, inverse=False):
    """Rows then columns, each with the line model (fft_ref.py:72-79)."""
    out = np.array(a, np.complex128)
    n = out.shape[0]
    for row in range(n):
        out[row, :] = dit_line(out[row, :], inverse)
    for col in range(n):
        out[:, col] = dit_line(out[:, col], inverse)
    return out


def is_bijective(n: int) -> bool:
    """Digit reversal is a permutation of [0, n) (fft_ref.py:82-85)."""
    t = digit_reverse_table(n)
    return bool(np.array_equal(np.sort(t), np.arange(n, dtype=np.uint32)))
