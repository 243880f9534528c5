"""FP64 restatement of reference/spectral2d.py on the GPU (torch complex128, cuFFT).

TEST INFRASTRUCTURE ONLY.  The long-run statistic tests compare the library's FP32
and split-precision paths with an FP64 run of the reference scheme at sizes and step
counts where the NumPy oracle (oracle/spectral_oracle.py) is too slow (4096^2, 5000
steps).  This class follows SpectralOracle operation for operation and is pinned
against it at small N by tests/test_gpu_long_runs.py::test_fp64_torch_matches_numpy_oracle.

Two guards the reference does not need at its own settings, both exact for the
library's configurations:
* out-of-band modes stay exactly zero (the integrating factor E(-dt/2) of an order-4
  hyperviscosity overflows beyond the dealias band, and inf * 0 would be NaN);
* the forcing is supplied per step as a sparse list of annulus cells.
"""
from __future__ import annotations

import math

import numpy as np

from oracle import wgsl_oracle as wo
from oracle.spectral_oracle import dealias_mask, wavenumbers


class Fp64Torch:
    def __init__(self, n, beta=0.0, mu=0.0, nu_h=0.0, hyper_p=1, device="cuda"):
        import torch
        self.torch = torch
        self.n = n
        self.dev = device
        k = torch.as_tensor(wavenumbers(n), dtype=torch.float64, device=device)
        self.kx = k[None, :].expand(n, n).contiguous()
        self.ky = k[:, None].expand(n, n).contiguous()
        self.k2 = self.kx ** 2 + self.ky ** 2
        self.k2_inv = torch.where(self.k2 > 0, 1.0 / torch.where(self.k2 > 0, self.k2, 1.0), 0.0)
        self.mask = torch.as_tensor(dealias_mask(n), device=device)
        lin_re = -mu - nu_h * self.k2 ** hyper_p
        lin_im = beta * self.kx * self.k2_inv
        self.lin = torch.complex(lin_re, lin_im)
        self.lin[0, 0] = complex(-mu, 0.0)
        self.partner = torch.as_tensor((-np.arange(n)) % n, device=device)
        self.w = torch.zeros((n, n), dtype=torch.complex128, device=device)
        self.t = 0.0

    # --- state
    def set_spectrum(self, w):
        self.w = self.torch.as_tensor(np.asarray(w), device=self.dev).to(self.torch.complex128)

    def set_vorticity(self, field):
        t = self.torch
        w = t.fft.fft2(t.as_tensor(np.asarray(field, np.float64), device=self.dev)) * self.mask
        w[0, 0] = 0.0
        self.w = w

    def spectrum_np(self):
        return self.w.cpu().numpy()

    # --- right-hand side (spectral2d.py:45-64)
    def nonlinear(self, w):
        t = self.torch
        uh = 1j * self.ky * self.k2_inv * w
        vh = -1j * self.kx * self.k2_inv * w
        a = t.fft.ifft2(w + 1j * uh)
        b = t.fft.ifft2(vh)
        omega, u, v = a.real, a.imag, b.real
        z = t.fft.fft2(t.complex(u * omega, v * omega))
        zm = t.conj(z[self.partner][:, self.partner])
        q1 = 0.5 * (z + zm)
        q2 = -0.5j * (z - zm)
        return (1j * self.kx * q1 + 1j * self.ky * q2) * self.mask

    def rhs(self, w, forcing):
        f = -self.nonlinear(w)
        return f if forcing is None else f + forcing

    def _apply(self, e, x):
        """E * x with E * 0 = 0 where E overflows (out-of-band modes)."""
        return self.torch.where(x == 0, self.torch.zeros_like(x), e * x)

    def factors(self, dt):
        """E(dt), E(dt/2), E(-dt/2) (spectral2d.py:73-74), kept for the last dt."""
        if getattr(self, "_fdt", None) != dt:
            t = self.torch
            self._f = (t.exp(self.lin * dt), t.exp(self.lin * (0.5 * dt)), t.exp(self.lin * (-0.5 * dt)))
            self._fdt = dt
        return self._f

    def step(self, dt, forcing=None):
        """spectral2d.py:76-90 with the RK rows of solver.js:11-15."""
        e_full, e_half, e_mhalf = self.factors(dt)
        w0 = self.w
        w1 = self._apply(e_full, w0 + dt * self.rhs(w0, forcing))
        w2 = 0.75 * self._apply(e_half, w0) + 0.25 * self._apply(e_mhalf, w1 + dt * self.rhs(w1, forcing))
        w3 = (1.0 / 3.0) * self._apply(e_full, w0) + (2.0 / 3.0) * self._apply(e_half, w2 + dt * self.rhs(w2, forcing))
        w3[0, 0] = 0.0
        self.w = w3
        self.t += dt

    # --- diagnostics (spectral2d.py:92-108), returned as NumPy float64
    def energy(self):
        return float(0.5 * (self.w.abs() ** 2 * self.k2_inv).sum() / self.n ** 4)

    def enstrophy(self):
        return float(0.5 * (self.w.abs() ** 2).sum() / self.n ** 4)

    def spectrum(self):
        t = self.torch
        nb = self.n // 2 + 1
        b = t.clamp(t.round(t.sqrt(self.k2)).long(), 0, self.n // 2)
        dens = 0.5 * self.w.abs() ** 2 * self.k2_inv / self.n ** 4
        e = t.zeros(nb, dtype=t.float64, device=self.dev).index_add_(0, b.reshape(-1), dens.reshape(-1))
        return e.cpu().numpy()

    def zonal_mean_u(self):
        t = self.torch
        uh = 1j * self.ky * self.k2_inv * self.w
        return t.fft.ifft2(uh).real.mean(dim=1).cpu().numpy()


class AnnulusForcing:
    """The stochastic annulus forcing of solver.wgsl:77-92 (wgsl_oracle.stochastic_forcing)
    in FP64, with the annulus cells found once: per step only the hashed phases of those
    cells are evaluated and scattered into a dense complex128 tensor."""

    def __init__(self, n, amp, k0, width, device="cuda"):
        import torch
        self.torch = torch
        self.n = n
        self.dev = device
        k = wavenumbers(n)
        kx = np.broadcast_to(k[None, :], (n, n))
        ky = np.broadcast_to(k[:, None], (n, n))
        k2 = kx * kx + ky * ky
        d = (np.sqrt(k2) - k0) / width
        env = np.exp(-(d * d))
        on = dealias_mask(n) & (k2 > 0) & (env > 1e-4)
        rows, cols = np.nonzero(on)
        kxs, kys = kx[rows, cols], ky[rows, cols]
        canon = (kys > 0) | ((kys == 0) & (kxs > 0))
        self.hr = np.where(canon, rows, (n - rows) % n).astype(np.uint32)
        self.hc = np.where(canon, cols, (n - cols) % n).astype(np.uint32)
        self.sgn = np.where(canon, 1.0, -1.0)
        self.base = amp * env[rows, cols] * float(wo.force_norm_f32(n))
        self.idx = torch.as_tensor(rows * n + cols, device=device)

    def __call__(self, step_index, dt):
        t = self.torch
        ph = 2.0 * math.pi * wo.hashf(self.hr * np.uint32(self.n) + self.hc, np.uint32(step_index)).astype(np.float64)
        amp = self.base / math.sqrt(max(dt, 1e-6))
        vals = amp * np.cos(ph) + 1j * (amp * self.sgn * np.sin(ph))
        out = t.zeros(self.n * self.n, dtype=t.complex128, device=self.dev)
        out[self.idx] = t.as_tensor(vals, device=self.dev)
        return out.reshape(self.n, self.n)
