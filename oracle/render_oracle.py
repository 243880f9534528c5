"""CPU restatement of the reference's fragment shader (src/shaders/render.wgsl:37-103)
-- TEST INFRASTRUCTURE ONLY: the checker for the headless render kernel.

PARITY UNPINNED: the WGSL runs only in a browser (no graphics stack here); this follows
its arithmetic in float32 with the repeat-wrapped bilinear sampling of the dye texture
and of the vorticity / velocity buffers.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def _bilinear(field, u, v):
    """field (n, n, c) sampled at normalised (u, v) with wrap (render.wgsl:37-59)."""
    n = field.shape[0]
    gx = u * f32(n) - f32(0.5)
    gy = v * f32(n) - f32(0.5)
    bx, by = np.floor(gx), np.floor(gy)
    fx, fy = (gx - bx)[..., None], (gy - by)[..., None]
    ix, iy = bx.astype(np.int64), by.astype(np.int64)
    a00 = field[iy % n, ix % n]
    a10 = field[iy % n, (ix + 1) % n]
    a01 = field[(iy + 1) % n, ix % n]
    a11 = field[(iy + 1) % n, (ix + 1) % n]
    mix = lambda a, b, t: a * (f32(1) - t) + b * t
    return mix(mix(a00, a10, fx), mix(a01, a11, fx), fy).astype(np.float32)


def _smoothstep(e0, e1, x):
    t = np.clip((x - f32(e0)) / f32(e1 - e0), 0, 1).astype(np.float32)
    return t * t * (f32(3) - f32(2) * t)


def _vort_color(t):
    a = np.clip(t, -1, 1)
    m = np.abs(a)
    hue = np.where((a > 0)[..., None], np.array([1.0, 0.40, 0.12], np.float32), np.array([0.16, 0.52, 1.0], np.float32))
    s = _smoothstep(0.0, 0.60, m)[..., None]
    base = np.array([0.035, 0.042, 0.062], np.float32) * (f32(1) - s) + hue * s
    w = (_smoothstep(0.70, 1.0, m) * f32(0.7))[..., None]
    return base * (f32(1) - w) + np.array([1.0, 0.95, 0.88], np.float32) * w


def _heat(t):
    x = np.clip(t, 0, 1)
    r = np.clip(f32(1.55) * x - f32(0.18), 0, 1)
    g = np.clip(f32(1.32) * x * x - f32(0.06), 0, 1)
    b = np.clip(f32(2.20) * x * x * x * (f32(1) - f32(0.55) * x) + f32(0.14) * x, 0, 1)
    return np.stack([r, g, b], -1) * f32(0.94) + np.array([0.03, 0.035, 0.055], np.float32)


def render(dye_rgba, omega, vel, mode, exposure, vort_scale, dye_gain, width, height):
    """dye_rgba (m, m, 4) float, omega (n, n), vel (n, n, 2) -> (height, width, 4) uint8, row 0 at the top."""
    px = np.arange(width, dtype=np.float32)
    py = np.arange(height, dtype=np.float32)
    u = ((px + f32(0.5)) / f32(width))[None, :].repeat(height, 0)
    v = (f32(1) - (py + f32(0.5)) / f32(height))[:, None].repeat(width, 1)
    dye = _bilinear(dye_rgba.astype(np.float32), u, v)[..., :3] * f32(dye_gain)
    om = _bilinear(omega.astype(np.float32)[..., None], u, v)[..., 0]
    t = np.clip(om * f32(vort_scale), -1, 1).astype(np.float32)
    if mode == 0:
        col = dye
    elif mode == 1:
        col = _vort_color(t)
    elif mode == 2:
        col = _vort_color(t) * (f32(0.30) + f32(0.70) * f32(exposure)) + dye * (f32(0.55) + f32(0.45) * np.abs(t))[..., None]
    else:
        w = _bilinear(vel.astype(np.float32), u, v)
        col = _heat(np.sqrt(w[..., 0] ** 2 + w[..., 1] ** 2) * f32(vort_scale) * f32(0.75))
    col = f32(1) - np.exp(-col * f32(exposure))
    col = np.power(np.clip(col, 0, 1), f32(0.4545))
    out = np.empty((height, width, 4), np.uint8)
    out[..., :3] = np.rint(np.clip(col, 0, 1) * 255).astype(np.uint8)
    out[..., 3] = 255
    return out
