"""NumPy restatement of the step's WGSL / JS-only arithmetic.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

PARITY UNPINNED: the reference ships no test, fixture or CPU implementation for
anything in this file (stochastic forcing, pointer forcing, CFL reduction,
fixed-point spectrum, seeding, dye painting and dye advection exist only as
WGSL shaders and browser JavaScript, which cannot run here).  Each function
restates the cited shader / script lines; the CUDA kernels are checked against
these restatements.

Float32 arithmetic is emulated with NumPy float32 operations (one rounding per
operation); the CUDA kernels may contract multiply-adds, so comparisons use
small tolerances, stated in the tests.  Integer hashing is bit-exact.
"""
from __future__ import annotations

import numpy as np

F32 = np.float32
U32 = np.uint32
TWO_PI_F32 = F32(6.28318530717958647)          # common.wgsl:5
HASH_SCALE = F32(2.3283064365386963e-10)       # common.wgsl:83


# ----------------------------------------------------------------------------- hashing
def hash1(x):
    """PCG-style u32 hash (common.wgsl:76-80; identical to hash32, solver.js:43-47)."""
    with np.errstate(over="ignore"):
        v = np.asarray(x, dtype=U32) * U32(747796405) + U32(2891336453)
        v = ((v >> ((v >> U32(28)) + U32(4))) ^ v) * U32(277803737)
        return (v >> U32(22)) ^ v


def hashf(a, b):
    """Uniform float in [0,1) from two u32 (common.wgsl:82-84)."""
    h = hash1(np.asarray(a, dtype=U32) ^ hash1(np.asarray(b, dtype=U32)))
    return h.astype(F32) * HASH_SCALE


# ----------------------------------------------------------------------------- grid helpers
def wn_f32(n):
    """wn(i) as f32 (common.wgsl:50-55)."""
    i = np.arange(n)
    return np.where(i < n // 2, i, i - n).astype(F32)


def kcut_f32(n):
    """KCUT constant, the f32 literal of n/3 (shaders.js:25)."""
    return F32(n / 3.0)


def force_norm_f32(n):
    """FORCE_NORM = 0.01 n^2 as an f32 literal (shaders.js:26)."""
    return F32(0.01 * n * n)


def in_band(n):
    k = wn_f32(n)
    b = np.abs(k) < kcut_f32(n)
    return b[:, None] & b[None, :]


def nu_h_from_rate(rate, n, hyper_p):
    """Solver.configure viscosity mapping, f32 result (solver.js:307,311)."""
    kcut = n / 3.0
    return F32(rate / kcut ** (2 * hyper_p)) if rate > 0 else F32(0.0)


# ----------------------------------------------------------------------------- stochastic forcing
def stochastic_forcing(n, force_amp, force_k, force_width, step_index, dt):
    """White-in-time annulus forcing added by ``assemble`` (solver.wgsl:77-92).

    Returns complex64 [n, n].  The envelope uses the square of
    ``(|k| - forceK)/forceWidth`` (the shader writes ``pow(x, 2.0)``; WGSL leaves
    ``pow`` of a negative base undefined, and the intended, symmetric annulus is
    the square).
    """
    out = np.zeros((n, n), np.complex64)
    force_amp, force_k, force_width = F32(force_amp), F32(force_k), F32(force_width)
    if not force_amp > 0:
        return out
    kx = wn_f32(n)[None, :] * np.ones((n, 1), F32)
    ky = wn_f32(n)[:, None] * np.ones((1, n), F32)
    k2 = kx * kx + ky * ky
    mask = in_band(n)
    d = (np.sqrt(k2) - force_k) / force_width
    env = np.exp(-(d * d)).astype(F32)
    on = mask & (k2 > 0) & (env > F32(1e-4))
    rows, cols = np.nonzero(on)
    kxs, kys = kx[rows, cols], ky[rows, cols]
    canon = (kys > 0) | ((kys == 0) & (kxs > 0))
    hr = np.where(canon, rows, (n - rows) % n).astype(U32)
    hc = np.where(canon, cols, (n - cols) % n).astype(U32)
    sgn = np.where(canon, F32(1.0), F32(-1.0)).astype(F32)
    ph = TWO_PI_F32 * hashf(hr * U32(n) + hc, U32(step_index))
    amp = force_amp * env[rows, cols] * force_norm_f32(n) / np.sqrt(np.maximum(F32(dt), F32(1e-6)))
    out[rows, cols] = (amp * np.cos(ph)).astype(F32) + 1j * (amp * sgn * np.sin(ph)).astype(F32)
    return out


# ----------------------------------------------------------------------------- pointer forcing
SPLAT_DTYPE = np.dtype([("x", F32), ("y", F32), ("dx", F32), ("dy", F32), ("r", F32),
                        ("g", F32), ("b", F32), ("radius", F32), ("amp", F32), ("dye_amp", F32)])


def _sep(a, b):
    """Periodic separation in [-1/2, 1/2) (common.wgsl:42-48)."""
    x = (a - b + F32(0.5)).astype(F32)
    return (x - np.floor(x) - F32(0.5)).astype(F32)


def pointer_force(n, splats):
    """Curl of a Gaussian body force from up to 8 splats (force.wgsl:5-27). Real f32 [n, n]."""
    idx = np.arange(n, dtype=F32)
    x = ((idx + F32(0.5)) / F32(n))[None, :] * np.ones((n, 1), F32)
    y = ((idx + F32(0.5)) / F32(n))[:, None] * np.ones((1, n), F32)
    total = np.zeros((n, n), F32)
    for s in splats[:8]:
        rx = _sep(x, F32(s["x"]))
        ry = _sep(y, F32(s["y"]))
        r2 = rx * rx + ry * ry
        sig2 = max(F32(s["radius"]) * F32(s["radius"]), F32(1e-8))
        g = np.exp(-r2 / sig2).astype(F32)
        term = F32(2.0) * F32(s["amp"]) * g * (F32(s["dx"]) * ry - F32(s["dy"]) * rx) / sig2
        total = total + np.where(r2 < F32(9.0) * sig2, term, F32(0.0)).astype(F32)
    return total


# ----------------------------------------------------------------------------- CFL reduction
def cfl_dt(u, v, n, cfl, dt_min, dt_max):
    """reduce_speed + reduce_dt (reduce.wgsl:22-63): returns (dt, max |u|+|v|) as f32."""
    speed = F32(np.max(np.abs(u.astype(F32)) + np.abs(v.astype(F32))))
    dx = F32(2.0 * np.pi / n)
    dt = F32(dt_max)
    if speed > F32(1e-8):
        dt = min(F32(dt_max), F32(cfl) * dx / speed)
    return F32(max(dt, F32(dt_min))), speed


# ----------------------------------------------------------------------------- diagnostics
def spectrum_fixed_point(w, n):
    """u32 fixed-point bins/totals as accumulated by spectrum.wgsl:19-39, decoded as solver.js:591-602.

    Each in-band cell contributes trunc(ene*1e8) to its bin, trunc(ene*1e6) to the
    energy and trunc(ens*1e6) to the enstrophy counter (u32 wrap-around).
    Returns (spectrum[n/2+1] float, energy, enstrophy).
    """
    w = np.asarray(w, np.complex64)
    nb = n // 2 + 1
    kx = wn_f32(n)[None, :] * np.ones((n, 1), F32)
    ky = wn_f32(n)[:, None] * np.ones((1, n), F32)
    k2 = kx * kx + ky * ky
    sel = in_band(n) & (k2 > 0)
    a = w[sel]
    n2 = F32(n) * F32(n)
    ens = F32(0.5) * (a.real * a.real + a.imag * a.imag) / (n2 * n2)
    ene = ens / k2[sel]
    b = np.minimum(np.floor(np.sqrt(k2[sel]) + F32(0.5)).astype(np.int64), nb - 1)
    bins = np.zeros(nb + 2, np.uint64)
    np.add.at(bins, b, (ene * F32(1e8)).astype(np.uint64))
    bins[nb] = np.sum((ene * F32(1e6)).astype(np.uint64))
    bins[nb + 1] = np.sum((ens * F32(1e6)).astype(np.uint64))
    bins = (bins % (1 << 32)).astype(np.uint32)
    return bins[:nb] / 1e8, bins[nb] / 1e6, bins[nb + 1] / 1e6


# ----------------------------------------------------------------------------- seeding
def fill_spectrum(n, k0, amplitude, seed):
    """Host spectral seeding ``Solver.fillSpectrum`` (solver.js:347-359, 384-418).

    Double-precision JS arithmetic stored to a Float32Array, then scaled in
    place (f32 * f64 -> f32).  Returns complex64 [n, n].
    """
    data = np.zeros((n, n), np.complex64)
    if not amplitude > 0:
        return data
    kcut = n / 3.0
    salt = int(hash1(np.uint32(seed & 0xFFFFFFFF)))
    k = np.arange(n)
    kx = np.where(k < n / 2, k, k - n).astype(np.float64)[None, :] * np.ones((n, 1))
    ky = np.where(k < n / 2, k, k - n).astype(np.float64)[:, None] * np.ones((1, n))
    rows = np.arange(n)[:, None] * np.ones((1, n), np.int64)
    cols = np.arange(n)[None, :] * np.ones((n, 1), np.int64)
    skip = ((kx == 0) & (ky == 0)) | (np.abs(kx) >= kcut) | (np.abs(ky) >= kcut)
    kr = np.hypot(kx, ky)
    env = kr * kr / (1.0 + (kr / k0) ** 8)
    amp = np.sqrt(env)
    canon = (ky > 0) | ((ky == 0) & (kx > 0))
    hr = np.where(canon, rows, (n - rows) % n)
    hc = np.where(canon, cols, (n - cols) % n)
    sgn = np.where(canon, 1.0, -1.0)
    h = hash1(((hr * n + hc).astype(np.uint64) & 0xFFFFFFFF).astype(U32) ^ U32(salt))
    phase = 2.0 * np.pi * h.astype(np.float64) / 4294967296.0
    re = np.where(skip, 0.0, amp * np.cos(phase)).astype(F32)
    im = np.where(skip, 0.0, sgn * amp * np.sin(phase)).astype(F32)
    total = float(np.sum(np.where(skip, 0.0, amp * amp)))
    rms = np.sqrt(total) / (n * n)
    if rms > 0:
        scale = amplitude / rms
        re = (re.astype(np.float64) * scale).astype(F32)
        im = (im.astype(np.float64) * scale).astype(F32)
    data.real = re
    data.imag = im
    return data


def seed_mask(src):
    """Dealias mask with k=0 removed on a transformed physical field (seed.wgsl:4-17)."""
    n = src.shape[0]
    out = np.where(in_band(n), src, 0).astype(np.complex64)
    out[0, 0] = 0
    return out


# ----------------------------------------------------------------------------- half floats
def to_half_bits(value):
    """JS ``toHalf`` (solver.js:20-41): f32 rounding, then mantissa TRUNCATION to binary16 bits."""
    f = np.asarray(value, dtype=F32)
    x = f.view(U32).astype(np.int64)
    sign = (x >> 16) & 0x8000
    exp = (x >> 23) & 0xFF
    mant = x & 0x7FFFFF
    out = np.zeros_like(x)
    nan_inf = exp == 255
    out = np.where(nan_inf, sign | 0x7C00 | np.where(mant != 0, 0x200, 0), out)
    e = exp - 127 + 15
    over = (~nan_inf) & (e >= 31)
    out = np.where(over, sign | 0x7C00, out)
    sub = (~nan_inf) & (~over) & (e <= 0)
    shift = np.clip(1 - e, 0, 63)
    sub_val = np.where(e < -10, sign, sign | (((mant | 0x800000) >> shift) >> 13))
    out = np.where(sub, sub_val, out)
    norm = (~nan_inf) & (~over) & (~sub)
    out = np.where(norm, sign | (e << 10) | (mant >> 13), out)
    return out.astype(np.uint16)


def half_bits_to_f32(bits):
    return np.asarray(bits, np.uint16).view(np.float16).astype(F32)


def paint_dye_bands(m):
    """'bands' dye pattern as binary16 bits [m, m, 4] (solver.js:446-473)."""
    warm = np.array([1.0, 0.45, 0.22])
    cool = np.array([0.28, 0.62, 1.0])
    fy = np.arange(m, dtype=np.float64) / m
    fx = np.arange(m, dtype=np.float64) / m
    band = 0.5 + 0.5 * np.tanh(6.0 * np.sin(fy * np.pi * 12.0))
    mix = 0.5 + 0.5 * np.sin(fx * np.pi * 2.0)
    out = np.zeros((m, m, 4), np.uint16)
    for c in range(3):
        val = band[:, None] * (warm[c] * mix[None, :] + cool[c] * (1.0 - mix[None, :])) * 0.9
        out[:, :, c] = to_half_bits(val.astype(F32))
    out[:, :, 3] = to_half_bits(np.float32(1.0))
    return out


# ----------------------------------------------------------------------------- dye advection
def _fma32(a, b, c):
    """a * b + c with one FP32 rounding, as the CUDA kernels' fused multiply-add: the
    product of two FP32 values is exact in FP64, the sum is rounded once to FP64 and then
    to FP32 (the two roundings can differ from one only when the FP64 sum lands exactly on
    an FP32 rounding midpoint, which these magnitudes make vanishingly rare)."""
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(F32)


def _lerp(a, b, t):
    """WGSL mix(a, b, t) as the kernels evaluate it: fma(b, t, a * (1 - t))."""
    one = F32(1.0)
    return _fma32(b, t, (a * (one - t)).astype(F32))


def _bilinear(tex, px, py, size):
    """Repeat-wrapped bilinear sample at normalised coords (software form of dye.wgsl:64,73,84-85),
    with the kernels' operation order (one fused multiply-add per interpolation)."""
    gx = (px * F32(size) - F32(0.5)).astype(F32)
    gy = (py * F32(size) - F32(0.5)).astype(F32)
    bx, by = np.floor(gx), np.floor(gy)
    fx, fy = (gx - bx).astype(F32), (gy - by).astype(F32)
    ix = bx.astype(np.int64) % size
    iy = by.astype(np.int64) % size
    ix1, iy1 = (ix + 1) % size, (iy + 1) % size
    fx = fx[..., None] if tex.ndim == 3 else fx
    fy = fy[..., None] if tex.ndim == 3 else fy
    t00, t10, t01, t11 = tex[iy, ix], tex[iy, ix1], tex[iy1, ix], tex[iy1, ix1]
    a = _lerp(t00, t10, fx)
    b = _lerp(t01, t11, fx)
    return _lerp(a, b, fy)


def _trace(px, py, vel, n, h):
    """Midpoint back-trace with bilinear velocity (dye.wgsl:20-45)."""
    v1 = _bilinear(vel, px, py, n) * F32(h)
    mx = (px - F32(0.5) * v1[..., 0] + F32(1.0)).astype(F32)
    my = (py - F32(0.5) * v1[..., 1] + F32(1.0)).astype(F32)
    mx, my = (mx - np.floor(mx)).astype(F32), (my - np.floor(my)).astype(F32)
    v2 = _bilinear(vel, mx, my, n) * F32(h)
    sx = (px - v2[..., 0] + F32(1.0)).astype(F32)
    sy = (py - v2[..., 1] + F32(1.0)).astype(F32)
    return (sx - np.floor(sx)).astype(F32), (sy - np.floor(sy)).astype(F32)


def dye_step(dye_bits, vel, dt, fade, splats=()):
    """BFECC + MacCormack-limited dye advection, one substep (dye.wgsl:58-113).

    ``dye_bits``: binary16 bits [m, m, 4]; ``vel``: f32 [n, n, 2] (u, v).
    Returns the new binary16 bits [m, m, 4] (round-to-nearest-even stores).
    """
    m = dye_bits.shape[0]
    n = vel.shape[0]
    src = half_bits_to_f32(dye_bits)
    vel = vel.astype(F32)
    c = np.arange(m, dtype=F32)
    px = ((c + F32(0.5)) / F32(m))[None, :] * np.ones((m, 1), F32)
    py = ((c + F32(0.5)) / F32(m))[:, None] * np.ones((1, m), F32)
    h = F32(dt) / TWO_PI_F32
    sx, sy = _trace(px, py, vel, n, h)
    fwd = _bilinear(src, sx, sy, m).astype(np.float16).astype(F32)          # advect_fwd
    bx, by = _trace(px, py, vel, n, -h)
    back = _bilinear(fwd, bx, by, m).astype(np.float16).astype(F32)         # advect_back
    a = _bilinear(src, sx, sy, m)                                           # advect_corr
    b = _bilinear(back, sx, sy, m)
    corr = (F32(1.5) * a - F32(0.5) * b).astype(F32)
    gx = (sx * F32(m) - F32(0.5)).astype(F32)
    gy = (sy * F32(m) - F32(0.5)).astype(F32)
    ix = np.floor(gx).astype(np.int64) % m
    iy = np.floor(gy).astype(np.int64) % m
    ix1, iy1 = (ix + 1) % m, (iy + 1) % m
    cs = [src[iy, ix], src[iy, ix1], src[iy1, ix], src[iy1, ix1]]
    lo = np.minimum(np.minimum(cs[0], cs[1]), np.minimum(cs[2], cs[3]))
    hi = np.maximum(np.maximum(cs[0], cs[1]), np.maximum(cs[2], cs[3]))
    res = (np.clip(corr, lo, hi) * F32(fade)).astype(F32)
    for s in list(splats)[:8]:
        rx = _sep(px, F32(s["x"]))
        ry = _sep(py, F32(s["y"]))
        sig2 = max(F32(s["radius"]) * F32(s["radius"]), F32(1e-8))
        r2 = rx * rx + ry * ry
        wgt = np.where(r2 < F32(9.0) * sig2, F32(s["dye_amp"]) * np.exp(-r2 / sig2), F32(0.0)).astype(F32)
        col = np.array([s["r"], s["g"], s["b"]], F32)
        res[..., :3] = (res[..., :3] + col[None, None, :] * wgt[..., None]).astype(F32)
    res[..., 3] = F32(1.0)
    return res.astype(np.float16).view(np.uint16)


# ----------------------------------------------------------------------------- band seed
def band_seed_spectrum(n, kmin, kmax, rms, seed):
    """Restatement of the library's band-limited seed (s2d_seed_band; no reference
    counterpart -- the benchmark configurations describe the field: complex Gaussian
    noise in kmin <= |k| <= kmax, Hermitian-symmetrised, dealiased, k = 0 removed, rms
    vorticity `rms`).  Cell (row, col) draws a complex Gaussian g by Box-Muller over
    two hash1 values of (seed, row*n + col), evaluated in FP64 and rounded to FP32;
    w = (g(k) + conj g(-k)) / 2 inside the band; then w *= rms / (sqrt(sum |w|^2) / n^2)
    in FP64 with one FP32 rounding.  Returns complex64 (n, n).
    """
    idx = np.arange(n * n, dtype=np.uint64).astype(U32)

    def gauss(i):
        h1 = hash1(i ^ hash1(U32(seed) ^ U32(0x68BC21EB)))
        h2 = hash1(h1 ^ U32(0x02E5BE93))
        u1 = (h1.astype(np.float64) + 0.5) * (1.0 / 4294967296.0)
        u2 = h2.astype(np.float64) * (1.0 / 4294967296.0)
        r = np.sqrt(-2.0 * np.log(u1))
        ang = np.pi * (2.0 * u2)
        return (r * np.cos(ang)).astype(F32), (r * np.sin(ang)).astype(F32)

    ax, ay = gauss(idx)
    row = (idx // U32(n)).astype(np.int64)
    col = (idx % U32(n)).astype(np.int64)
    pidx = (((n - row) % n) * n + ((n - col) % n)).astype(np.uint64).astype(U32)
    bx, by = gauss(pidx)
    kx = np.where(col < n // 2, col, col - n).astype(F32)
    ky = np.where(row < n // 2, row, row - n).astype(F32)
    kr = np.sqrt(kx * kx + ky * ky).astype(F32)
    kcut = F32(n / 3.0)
    inside = (kr != 0) & (kr >= F32(kmin)) & (kr <= F32(kmax)) & (np.abs(kx) < kcut) & (np.abs(ky) < kcut)
    wx = np.where(inside, F32(0.5) * (ax + bx), F32(0.0)).astype(F32)
    wy = np.where(inside, F32(0.5) * (ay - by), F32(0.0)).astype(F32)
    total = np.sum(wx.astype(np.float64) ** 2 + wy.astype(np.float64) ** 2)
    cur = np.sqrt(total) / (float(n) * float(n))
    sc = rms / cur if cur > 0 else 1.0
    out = (wx.astype(np.float64) * sc).astype(F32) + 1j * (wy.astype(np.float64) * sc).astype(F32)
    return out.astype(np.complex64).reshape(n, n)
