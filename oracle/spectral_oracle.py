"""FP64 restatement of the reference solver ``reference/spectral2d.py``.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Pinned against the
golden vectors under ``tests/golden/`` (made by ``tests/golden/make_golden.py``
from the reference's ``tests/fixtures.json`` and from ``reference/spectral2d.py``
itself).

Layout: spectral arrays are complex128 ``[row, col]`` with ``row`` the y index
(``ky = wn(row)``) and ``col`` the x index (``kx = wn(col)``), the same layout
as the reference (spectral2d.py:16-18).
"""
from __future__ import annotations

import numpy as np

TWO_PI = 2.0 * np.pi


def wavenumbers(n: int) -> np.ndarray:
    """Signed integer wavenumber of each FFT index (spectral2d.py:16, common.wgsl:50-55)."""
    i = np.arange(n)
    return np.where(i < n // 2, i, i - n).astype(np.float64)


def dealias_mask(n: int) -> np.ndarray:
    """2/3-rule mask ``|kx| < n/3 and |ky| < n/3`` (spectral2d.py:22-23, common.wgsl:69-74)."""
    k = wavenumbers(n)
    kcut = n / 3.0
    band = np.abs(k) < kcut
    return band[:, None] & band[None, :]


class SpectralOracle:
    """Integrating-factor SSP-RK3 vorticity solver on the doubly periodic beta-plane.

    Constructor arguments follow ``Spectral2D.__init__`` (spectral2d.py:7-31):
    ``tau`` is the damping time at the dealias cutoff, so
    ``nu_h = 1 / (tau * kcut**(2p))`` (spectral2d.py:24); ``nu_h`` may also be
    passed directly.
    """

    def __init__(self, n=256, beta=0.0, mu=0.0, tau=None, hyper_p=4, cfl=0.4,
                 dt_max=0.05, nu_h=None):
        self.n = int(n)
        self.beta = float(beta)
        self.mu = float(mu)
        self.hyper_p = int(hyper_p)
        self.cfl = float(cfl)
        self.dt_max = float(dt_max)
        self.dx = TWO_PI / n
        k = wavenumbers(n)
        self.kx = np.broadcast_to(k[None, :], (n, n)).copy()
        self.ky = np.broadcast_to(k[:, None], (n, n)).copy()
        self.k2 = self.kx ** 2 + self.ky ** 2
        safe = np.where(self.k2 > 0, self.k2, 1.0)
        self.k2_inv = np.where(self.k2 > 0, 1.0 / safe, 0.0)
        kcut = n / 3.0
        self.mask = dealias_mask(n)
        if nu_h is not None:
            self.nu_h = float(nu_h)
        else:
            self.nu_h = 0.0 if tau is None else 1.0 / (tau * kcut ** (2 * hyper_p))
        # linear operator, spectral2d.py:26-27 (k=0 keeps only the drag)
        self.lin = (-self.mu - self.nu_h * self.k2 ** self.hyper_p
                    + 1j * self.beta * self.kx * self.k2_inv)
        self.lin[0, 0] = -self.mu
        # conjugate-partner index -k, spectral2d.py:31
        self.partner = (-np.arange(n)) % n
        self.w = np.zeros((n, n), np.complex128)
        self.t = 0.0

    # --- state -----------------------------------------------------------------
    def set_vorticity(self, field):
        """Physical field -> masked spectrum with k=0 removed (spectral2d.py:33-35)."""
        w = np.fft.fft2(np.asarray(field, np.float64)) * self.mask
        w[0, 0] = 0.0
        self.w = w.astype(np.complex128)

    def vorticity(self):
        return np.fft.ifft2(self.w).real

    def velocity_hat(self, w):
        """u_hat = i ky w/k^2, v_hat = -i kx w/k^2 (spectral2d.py:41-42, 46-47)."""
        uh = 1j * self.ky * self.k2_inv * w
        vh = -1j * self.kx * self.k2_inv * w
        return uh, vh

    def velocity(self):
        uh, vh = self.velocity_hat(self.w)
        return np.fft.ifft2(uh).real, np.fft.ifft2(vh).real

    # --- right-hand side ---------------------------------------------------------
    def packs(self, w):
        """Two-for-one packing: packA = w + i u_hat, packB = v_hat (spectral2d.py:45-48)."""
        uh, vh = self.velocity_hat(w)
        return w + 1j * uh, vh

    def physical_fields(self, w):
        """(omega, u, v) from two complex inverse transforms (spectral2d.py:45-50)."""
        pa, pb = self.packs(w)
        a = np.fft.ifft2(pa)
        b = np.fft.ifft2(pb)
        return a.real, a.imag, b.real

    def product_spectrum(self, w):
        """Z = FFT2(u*omega + i v*omega) (spectral2d.py:53-54)."""
        omega, u, v = self.physical_fields(w)
        return np.fft.fft2(u * omega + 1j * (v * omega))

    def unpack_nonlinear(self, z):
        """Hermitian unpack of Z and the dealiased advection term (spectral2d.py:55-58)."""
        zm = np.conj(z[np.ix_(self.partner, self.partner)])
        q1 = 0.5 * (z + zm)
        q2 = -0.5j * (z - zm)
        return (1j * self.kx * q1 + 1j * self.ky * q2) * self.mask

    def nonlinear(self, w):
        return self.unpack_nonlinear(self.product_spectrum(w))

    def rhs(self, w, forcing=None):
        """f = -N(w) + forcing (spectral2d.py:60-64)."""
        f = -self.nonlinear(w)
        if forcing is not None:
            f = f + forcing
        return f

    # --- time stepping -------------------------------------------------------------
    def timestep(self):
        """Advective CFL dt from the current state (spectral2d.py:66-71)."""
        u, v = self.velocity()
        speed = float(np.max(np.abs(u) + np.abs(v)))
        if speed <= 1e-12:
            return self.dt_max
        return min(self.dt_max, self.cfl * self.dx / speed)

    def factor(self, s):
        """Integrating factor E(s) = exp(L s) (spectral2d.py:73-74)."""
        return np.exp(self.lin * s)

    def step(self, dt=None, forcing=None):
        """One SSP-RK3 step with the linear part integrated exactly (spectral2d.py:76-90).

        Stage coefficients [cA, a, cB, b]: wout = cA E(a dt) w0 + cB E(b dt) (wcur + dt f)
        with rows [0,0,1,1], [3/4,1/2,1/4,-1/2], [1/3,1,2/3,1/2] (solver.js:11-15).
        """
        if dt is None:
            dt = self.timestep()
        w0 = self.w
        e_full = self.factor(dt)
        e_half = self.factor(0.5 * dt)
        e_mhalf = self.factor(-0.5 * dt)
        w1 = e_full * (w0 + dt * self.rhs(w0, forcing))
        w2 = 0.75 * e_half * w0 + 0.25 * e_mhalf * (w1 + dt * self.rhs(w1, forcing))
        w3 = (1.0 / 3.0) * e_full * w0 + (2.0 / 3.0) * e_half * (w2 + dt * self.rhs(w2, forcing))
        w3[0, 0] = 0.0
        self.w = w3
        self.t += dt
        return dt

    # --- diagnostics ---------------------------------------------------------------
    def energy(self):
        """E = 1/2 sum |w|^2/k^2 / n^4 (spectral2d.py:92-93)."""
        return 0.5 * float(np.sum(np.abs(self.w) ** 2 * self.k2_inv)) / self.n ** 4

    def enstrophy(self):
        """Z = 1/2 sum |w|^2 / n^4 (spectral2d.py:95-96)."""
        return 0.5 * float(np.sum(np.abs(self.w) ** 2)) / self.n ** 4

    def spectrum(self):
        """Radial energy spectrum in bins round(|k|), n/2+1 bins (spectral2d.py:98-104)."""
        nb = self.n // 2 + 1
        b = np.clip(np.round(np.sqrt(self.k2)).astype(np.int64), 0, self.n // 2)
        dens = 0.5 * np.abs(self.w) ** 2 * self.k2_inv / self.n ** 4
        e = np.bincount(b.ravel(), weights=dens.ravel(), minlength=nb)
        return np.arange(nb), e[:nb]

    def zonal_mean_u(self):
        """Mean over x of u at each y row (spectral2d.py:106-108)."""
        u, _ = self.velocity()
        return u.mean(axis=1)


def random_field(n, k0=14.0, seed=0, amplitude=1.0):
    """Band-limited random physical field with unit-normalised std (spectral2d.py:111-123)."""
    rng = np.random.default_rng(seed)
    k = wavenumbers(n)
    k2 = k[None, :] ** 2 + k[:, None] ** 2
    kr = np.sqrt(k2)
    env = np.where(k2 > 0, kr ** 2 / (1.0 + (kr / k0) ** 8), 0.0)
    phase = rng.uniform(0, TWO_PI, (n, n))
    field = np.fft.ifft2(np.sqrt(env) * np.exp(1j * phase)).real
    field = field - field.mean()
    return amplitude * field / np.std(field)


def band_noise_spectrum(n, kmin, kmax, seed, rms=1.0):
    """Seeded complex Gaussian spectrum in ``kmin <= |k| <= kmax``, Hermitian, rms vorticity ``rms``.

    This is the initial condition of the benchmark workloads (free decay at 256^2,
    the ensembles): complex Gaussian noise kept in the band, Hermitian-symmetrised
    by taking the spectrum of its real part, dealias-masked, k=0 removed, then
    scaled so that the physical vorticity has the requested rms.
    """
    rng = np.random.default_rng(seed)
    k = wavenumbers(n)
    kr = np.sqrt(k[None, :] ** 2 + k[:, None] ** 2)
    noise = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    spec = np.where((kr >= kmin) & (kr <= kmax), noise, 0.0)
    field = np.fft.ifft2(spec).real
    w = np.fft.fft2(field) * dealias_mask(n)
    w[0, 0] = 0.0
    cur = np.sqrt(np.sum(np.abs(w) ** 2)) / (n * n)
    if cur > 0:
        w *= rms / cur
    return w
