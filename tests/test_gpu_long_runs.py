"""Long-run statistics of the benchmark configurations against an FP64 run.

The library's FP32 step (and the split-precision tensor-core steps where the grid
size has one) is run as each configuration is written, and its radial energy
spectrum, energy, enstrophy, zonal-mean u(y) and state are compared with an FP64 run
of the reference scheme (reference/spectral2d.py:76-108) from the same FP32 initial
bits.  The FP64 runs use tests/fp64_torch.py (torch complex128 on the GPU), pinned
against the NumPy oracle at small N by the first test.  Statistics are computed in
FP64 from the states each solver produced.
"""
import numpy as np
import pytest

from conftest import rel_l2
from fp64_torch import AnnulusForcing, Fp64Torch
from gpu_helpers import config, current_state, load_state, rate_for, set_fixed_dt
from oracle.spectral_oracle import SpectralOracle, random_field, wavenumbers

pytestmark = pytest.mark.gpu

FFTS = ["fp32", "tc-f16", "tc-bf16"]


def _solver(pkg, n, fft):
    """A Solver of this FFT path, or skip where the path has no kernel for size n."""
    try:
        return pkg.Solver.create(n=n, dyeScale=1, fft=fft)
    except pkg.S2DError as e:
        if e.status == -2:
            pytest.skip(f"fft={fft} has no kernel at {n}^2")
        raise


def _stats(w, n):
    """FP64 statistics of a spectral state (spectral2d.py:92-108)."""
    w = np.asarray(w, np.complex128)
    k = wavenumbers(n)
    kx, ky = k[None, :], k[:, None]
    k2 = kx ** 2 + ky ** 2
    k2i = np.where(k2 > 0, 1.0 / np.where(k2 > 0, k2, 1.0), 0.0)
    dens = 0.5 * np.abs(w) ** 2 * k2i / n ** 4
    b = np.clip(np.round(np.sqrt(k2)).astype(np.int64), 0, n // 2)
    spec = np.bincount(b.ravel(), weights=dens.ravel(), minlength=n // 2 + 1)[: n // 2 + 1]
    uh = 1j * ky * k2i * w
    zonal = np.fft.ifft2(uh).real.mean(axis=1)
    return {"energy": float(dens.sum()), "enstrophy": float(0.5 * np.sum(np.abs(w) ** 2) / n ** 4),
            "spectrum": spec, "zonal": zonal}


def _errors(got, want):
    g, r = _stats(got, got.shape[0]), _stats(want, want.shape[0])
    out = {"state": rel_l2(got, want),
           "energy": abs(g["energy"] / r["energy"] - 1.0),
           "enstrophy": abs(g["enstrophy"] / r["enstrophy"] - 1.0),
           "spectrum": float(np.linalg.norm(g["spectrum"] - r["spectrum"]) / np.linalg.norm(r["spectrum"]))}
    zn = np.linalg.norm(r["zonal"])
    out["zonal"] = float(np.linalg.norm(g["zonal"] - r["zonal"]) / zn) if zn > 0 else 0.0
    return out


def _report(name, fft, err):
    print(f"\n[long-run] {name} fft={fft} " + " ".join(f"{k}={v:.3e}" for k, v in err.items()))


def _run_fixed(s, steps, dt, chunk=250):
    """`steps` fused RK3 steps at the fixed `dt` (no CFL, no dye), each substep with its own
    forcing phase (stepIndex 0, 1, 2, ...).  The solver is primed first: priming runs the
    CFL reduction, so the fixed dt is written after it."""
    s.encodePrime()
    set_fixed_dt(s, dt)
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        s.step(k, dye=False, reduce=False, graph=False, relatch=True)
        done += k
    s.synchronize()


def test_fp64_torch_matches_numpy_oracle():
    """Pin of the FP64 GPU restatement: 10 steps at 64^2 with beta, hyperviscosity, drag
    and the stochastic forcing, against oracle.spectral_oracle."""
    n, dt = 64, 5e-3
    nu_h = 1.0 / (n / 3.0) ** 8
    ref = SpectralOracle(n=n, beta=7.0, mu=0.02, nu_h=nu_h, hyper_p=4)
    ref.set_vorticity(random_field(n, k0=8, seed=5, amplitude=2.0))
    gpu = Fp64Torch(n, beta=7.0, mu=0.02, nu_h=nu_h, hyper_p=4)
    gpu.set_spectrum(ref.w)
    forcing = AnnulusForcing(n, 0.1, 10.0, 2.0)
    for k in range(10):
        f = forcing(k, dt)
        ref.step(dt=dt, forcing=f.cpu().numpy())
        gpu.step(dt, f)
    assert rel_l2(gpu.spectrum_np(), ref.w) <= 1e-12
    assert abs(gpu.energy() / ref.energy() - 1) <= 1e-12
    assert np.allclose(gpu.spectrum(), ref.spectrum()[1], rtol=1e-11, atol=0)
    assert np.allclose(gpu.zonal_mean_u(), ref.zonal_mean_u(), rtol=0, atol=1e-12 * np.max(np.abs(ref.zonal_mean_u())))


def test_annulus_forcing_matches_restatement():
    """The FP64 forcing is the FP32 restatement's forcing to FP32 rounding."""
    from oracle.wgsl_oracle import stochastic_forcing
    n, dt = 128, 2e-3
    f64 = AnnulusForcing(n, 5e-2, 20.0, 3.0)(17, dt).cpu().numpy()
    f32 = stochastic_forcing(n, 5e-2, 20.0, 3.0, 17, dt)
    assert np.array_equal(f64 != 0, f32 != 0)
    assert rel_l2(f32, f64) <= 1e-6


# ---------------------------------------------------------------- configuration 1
@pytest.mark.parametrize("fft", FFTS)
def test_config1_free_decay_256(pkg, fft):
    """256^2, band 6 <= |k| <= 10 rms 1 (seed 0), nu = 1e-3 (p = 1), no forcing,
    dt = 2e-3 fixed, 1000 steps."""
    n, nu, dt, steps = 256, 1e-3, 2e-3, 1000
    s = _solver(pkg, n, fft)
    try:
        s.configure(config(viscosity=rate_for(nu, n, 1), hyperP=1))
        s.seedBand(6.0, 10.0, rms=1.0, seed=0)
        w0 = current_state(s)
        nu_h = float(s.paramsF[2])
        _run_fixed(s, steps, dt)
        got = current_state(s)
    finally:
        s.destroy()
    ref = Fp64Torch(n, nu_h=nu_h, hyper_p=1)
    ref.set_spectrum(w0)
    for _ in range(steps):
        ref.step(dt)
    err = _errors(got, ref.spectrum_np())
    _report("config1", fft, err)
    # measured on a B200, FP32: state 3.8e-6, energy 3.1e-6, enstrophy 3.0e-6, spectrum 3.9e-6
    bound = {"fp32": 1.2e-5, "tc-f16": 3e-5, "tc-bf16": 1e-4}[fft]
    assert err["state"] <= bound
    assert err["spectrum"] <= bound
    assert err["energy"] <= bound and err["enstrophy"] <= bound


@pytest.mark.parametrize("fft", FFTS)
def test_config1_taylor_green_256(pkg, fft):
    """Taylor-Green omega = 6 cos 2x cos 2y at 256^2, nu = 1e-3: the Jacobian vanishes
    (the state stays the single mode) and the mode decays as exp(-nu |k|^2 t)."""
    # measured FP32: Jacobian 5.7e-6, decay rate 5.7e-6 over 1000 steps; BF16 split: Jacobian 2.6e-5
    b = {"fp32": 2e-5, "tc-f16": 5e-5, "tc-bf16": 1e-4}[fft]
    _taylor_green(pkg, 256, 1000, fft, jac_bound=b, rate_bound=b)


# ---------------------------------------------------------------- configuration 2
@pytest.mark.parametrize("n", [1024, 2048])
def test_config2_forced_inverse_cascade(pkg, n):
    """Forced inverse cascade at 1024^2 and 2048^2, every FFT path against one FP64 run:
    white-in-time forcing |k| = 64 +- 2 at amplitude 0.1, order-4 hyperviscosity at damping
    rate 1 at the cutoff (the written nu4 = 1e-16 overflows E(-dt/2) in FP32 at 1024^2),
    drag 1e-2, beta 0, the benchmark's band seed (4 <= |k| <= 12, rms 1), dt = 5e-4 fixed
    (inside the CFL 0.5 limit of this flow; a fixed dt keeps the forcing amplitude, which
    scales as dt^-1/2, identical between the runs), 2000 steps."""
    dt, steps = 5e-4, 2000
    cfg = config(drag=1e-2, viscosity=1.0, hyperP=4, forceAmp=0.1, forceK=64.0, forceWidth=2.0)
    got, w0, nu_h = {}, None, None
    for fft in FFTS:
        s = pkg.Solver.create(n=n, dyeScale=1, fft=fft)
        try:
            s.configure(cfg)
            s.seedBand(4.0, 12.0, rms=1.0, seed=1)
            w = current_state(s)
            if w0 is None:
                w0, nu_h = w, float(s.paramsF[2])
            assert np.array_equal(w, w0)
            _run_fixed(s, steps, dt)
            got[fft] = current_state(s)
        finally:
            s.destroy()
    ref = Fp64Torch(n, mu=1e-2, nu_h=nu_h, hyper_p=4)
    ref.set_spectrum(w0)
    forcing = AnnulusForcing(n, 0.1, 64.0, 2.0)
    for k in range(steps):
        ref.step(dt, forcing(k, dt))
    want = ref.spectrum_np()
    del ref
    bounds = {"fp32": 2e-5, "tc-f16": 5e-5, "tc-bf16": 2e-4}
    for fft in FFTS:
        err = _errors(got[fft], want)
        _report(f"config2 n={n}", fft, err)
        for key in ("state", "energy", "enstrophy", "spectrum"):
            assert err[key] <= bounds[fft], f"{fft} {key} {err[key]:.3e}"


# ---------------------------------------------------------------- configuration 4
@pytest.mark.parametrize("fft", FFTS)
def test_config4_beta_plane_4096(pkg, fft):
    """4096^2 beta-plane: beta = 10, stochastic forcing |k| = 128 +- 3 at amplitude 5e-2,
    order-4 hyperviscosity at damping rate 1 at the cutoff (the written nu4 = 1e-20
    makes E(-dt/2) overflow FP32 inside the band), drag 5e-3, from rest, dt = 2e-4 fixed,
    1000 steps: zonal-mean u(y) and the radial spectrum against FP64."""
    n, dt, steps = 4096, 2e-4, 1000
    cfg = config(beta=10.0, drag=5e-3, viscosity=1.0, hyperP=4, forceAmp=5e-2, forceK=128.0, forceWidth=3.0)
    s = _solver(pkg, n, fft)
    try:
        s.configure(cfg)
        load_state(s, np.zeros((n, n), np.complex64))
        nu_h = float(s.paramsF[2])
        _run_fixed(s, steps, dt)
        got = current_state(s)
    finally:
        s.destroy()
    ref = Fp64Torch(n, beta=10.0, mu=5e-3, nu_h=nu_h, hyper_p=4)
    forcing = AnnulusForcing(n, 5e-2, 128.0, 3.0)
    for k in range(steps):
        ref.step(dt, forcing(k, dt))
    want = ref.spectrum_np()
    del ref
    err = _errors(got, want)
    _report("config4", fft, err)
    # measured FP32: state 1.7e-6, zonal 1.2e-6, spectrum 2.4e-7
    bound = {"fp32": 1e-5, "tc-f16": 5e-5, "tc-bf16": 2e-4}[fft]
    assert err["zonal"] <= bound
    assert err["spectrum"] <= bound
    assert err["state"] <= bound


# ---------------------------------------------------------------- configuration 5
def _taylor_green(pkg, n, steps, fft, jac_bound, rate_bound, nu=1e-3, dt=2e-3):
    xs = np.arange(n) * 2 * np.pi / n
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    s = _solver(pkg, n, fft)
    try:
        s.configure(config(viscosity=rate_for(nu, n, 1), hyperP=1))
        s.seedPhysical(6.0 * np.cos(2 * gx) * np.cos(2 * gy))
        w0 = current_state(s).astype(np.complex128)
        nu_h = float(s.paramsF[2])
        _run_fixed(s, steps, dt)
        w1 = current_state(s).astype(np.complex128)
    finally:
        s.destroy()
    decay = np.exp(-nu_h * 8.0 * dt * steps)
    jac = float(np.max(np.abs(w1 - decay * w0)) / np.max(np.abs(decay * w0)))
    rate = abs(abs(w1[2, 2] / w0[2, 2]) / decay - 1.0)
    print(f"\n[long-run] taylor-green n={n} steps={steps} fft={fft} jacobian={jac:.3e} decay_rate={rate:.3e}")
    assert jac <= jac_bound
    assert rate <= rate_bound


@pytest.mark.parametrize("fft", FFTS)
def test_config5a_taylor_green_512(pkg, fft):
    """512^2 Taylor-Green, nu = 1e-3, 5000 steps of dt = 2e-3 (t = 10)."""
    # measured FP32: Jacobian 6.7e-6, decay rate 6.7e-6 over 5000 steps
    # tc-f16: Jacobian 1.7e-5, decay 6.6e-6; tc-bf16: 1.6e-4 both (16-bit operands over 5000 steps)
    b = {"fp32": 2e-5, "tc-f16": 5e-5, "tc-bf16": 5e-4}[fft]
    _taylor_green(pkg, 512, 5000, fft, jac_bound=b, rate_bound=b)


def _compare_run(pkg, name, n, fft, field, nu, dt, steps, bounds):
    s = _solver(pkg, n, fft)
    try:
        s.configure(config(viscosity=rate_for(nu, n, 1) if nu > 0 else 0.0, hyperP=1))
        s.seedPhysical(field)
        w0 = current_state(s)
        nu_h = float(s.paramsF[2])
        _run_fixed(s, steps, dt)
        got = current_state(s)
    finally:
        s.destroy()
    ref = Fp64Torch(n, nu_h=nu_h, hyper_p=1)
    ref.set_spectrum(w0)
    e0, z0 = ref.energy(), ref.enstrophy()
    for _ in range(steps):
        ref.step(dt)
    err = _errors(got, ref.spectrum_np())
    _report(name, fft, err)
    if nu == 0:
        # the FP64 run's own conservation (dealiased Galerkin system; RK3 time error only)
        print(f"[long-run] {name} fp64 energy drift {abs(ref.energy() / e0 - 1):.3e} "
              f"enstrophy drift {abs(ref.enstrophy() / z0 - 1):.3e}")
    for k, b in bounds[fft].items():
        assert err[k] <= b, f"{name} {fft}: {k} error {err[k]:.3e} > {b:.1e}"


@pytest.mark.parametrize("fft", FFTS)
def test_config5b_double_shear_layer_512(pkg, fft):
    """Double shear layer at 512^2: u = tanh((y - pi/2)/d) for y <= pi, tanh((3pi/2 - y)/d)
    above, d = 30/N * 2 pi, v = 0.05 sin x, nu = 5e-5, to t = 8 (1600 steps of 5e-3)."""
    n = 512
    d = 30.0 / n * 2 * np.pi
    xs = np.arange(n) * 2 * np.pi / n
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    lower = gy <= np.pi
    dudy = np.where(lower, 1.0 / np.cosh((gy - np.pi / 2) / d) ** 2 / d,
                    -1.0 / np.cosh((1.5 * np.pi - gy) / d) ** 2 / d)
    omega = 0.05 * np.cos(gx) - dudy          # dv/dx - du/dy
    # the roll-up amplifies round-off: measured FP32 at t = 8: state 7.1e-5, energy 5.2e-5,
    # enstrophy 3.7e-5, spectrum 5.5e-5
    bounds = {"fp32": {"energy": 2e-4, "enstrophy": 2e-4, "spectrum": 2e-4},
              "tc-f16": {"energy": 1e-3, "enstrophy": 1e-3, "spectrum": 1e-3},
              "tc-bf16": {"energy": 1e-4, "enstrophy": 1e-3, "spectrum": 1e-2}}
    _compare_run(pkg, "config5b", n, fft, omega, 5e-5, 5e-3, 1600, bounds)


@pytest.mark.parametrize("fft", FFTS)
def test_config5c_vortex_pair_512(pkg, fft):
    """Two like-signed Gaussian vortices at 512^2, core 0.22, separation 0.9, nu = 0,
    2000 steps of 5e-3 (t = 10)."""
    n = 512
    xs = np.arange(n) * 2 * np.pi / n
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    a = 0.22
    omega = np.zeros((n, n))
    for cx in (np.pi - 0.45, np.pi + 0.45):
        omega += np.exp(-((gx - cx) ** 2 + (gy - np.pi) ** 2) / a ** 2)
    # measured FP32: state 1.6e-6, energy 1.3e-8, enstrophy 2.9e-7, spectrum 2.8e-7 (the FP64
    # run itself drifts 5.5e-8 / 2.4e-7: RK3 time error of the inviscid system)
    bounds = {"fp32": {"energy": 1e-6, "enstrophy": 1e-6, "spectrum": 1e-5, "state": 1e-5},
              "tc-f16": {"energy": 1e-5, "enstrophy": 1e-5, "spectrum": 1e-4, "state": 1e-3},
              "tc-bf16": {"energy": 1e-4, "enstrophy": 1e-4, "spectrum": 1e-3, "state": 1e-2}}
    _compare_run(pkg, "config5c", n, fft, omega, 0.0, 5e-3, 2000, bounds)
