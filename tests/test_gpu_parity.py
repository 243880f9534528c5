"""Parity of the CUDA path with the oracle: tables, FFTs, the fused RK3 step,
forcing, CFL reduction, seeding, and the Taylor-Green invariants."""
import numpy as np
import pytest

from conftest import rel_l2, rel_linf
from gpu_helpers import config, current_state, load_state, rate_for, set_fixed_dt
from oracle import fft_oracle as fo
from oracle import wgsl_oracle as wo
from oracle.spectral_oracle import SpectralOracle, dealias_mask, random_field, wavenumbers

pytestmark = pytest.mark.gpu

SIZES = [32, 64, 128, 256, 512, 1024, 2048, 4096]


# ---------------------------------------------------------------- bit-exact tables
@pytest.mark.parametrize("n", [2, 8, 32, 128, 512, 2048, 4, 16, 64, 256, 1024, 4096])
def test_digit_reverse_bit_exact(pkg, fft_golden, n):
    assert np.array_equal(pkg.digitReverseTable(n), fft_golden[f"rev_{n}"])


@pytest.mark.parametrize("n", SIZES)
def test_wavenumbers_and_mask_bit_exact(pkg, n):
    wn = pkg.wavenumberTable(n)
    assert wn.dtype == np.float32 and np.array_equal(wn, wavenumbers(n).astype(np.float32))
    assert np.array_equal(wn.view(np.uint32), wo.wn_f32(n).view(np.uint32))
    assert np.array_equal(pkg.dealiasMaskTable(n).astype(bool), dealias_mask(n))


# ---------------------------------------------------------------- FFT at every size
@pytest.mark.parametrize("n", SIZES)
def test_fft2_matches_numpy(pkg, n):
    rng = np.random.default_rng(n)
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.setBuffer("packB", a)
        s.fft.forward(None, "packB")
        fwd = s.getBuffer("packB")
        ref = np.fft.fft2(a.astype(np.complex128))
        assert rel_l2(fwd, ref) <= 2e-7 * np.log2(n) + 5e-7
        s.fft.inverse(None, "packB")
        back = s.getBuffer("packB")
        assert rel_l2(back, a) <= 2e-7 * np.log2(n) + 5e-7
    finally:
        s.destroy()


def test_fft_unregistered_buffer_throws(pkg):
    s = pkg.Solver.create(n=64, dyeScale=1)
    try:
        with pytest.raises(pkg.S2DError) as ei:
            s.fft.forward(None, "state0")
        assert ei.value.status == -6                                   # fft.js:84
    finally:
        s.destroy()


# ---------------------------------------------------------------- fused step vs FP64 oracle
CASES = [
    # n, beta, mu, nu_h, p, dt, amplitude
    (64, 5.0, 0.01, 1e-12, 4, 0.01, 2.0),
    (128, 12.0, 0.0, 0.0, 4, 2e-3, 6.0),
    (256, 0.0, 0.0, 1e-3, 1, 2e-3, 1.0),
    (512, 10.0, 5e-3, 1e-20, 4, 1e-3, 8.0),
    (1024, 0.0, 1e-2, 1.0 / (1024 / 3.0) ** 8, 4, 1e-3, 8.0),
]


@pytest.mark.parametrize("case", CASES, ids=[f"n{c[0]}" for c in CASES])
def test_fused_step_vs_oracle(pkg, case):
    n, beta, mu, nu_h, p, dt, amp = case
    ref = SpectralOracle(n=n, beta=beta, mu=mu, nu_h=nu_h, hyper_p=p)
    ref.set_vorticity(random_field(n, k0=n / 8, seed=n, amplitude=amp))
    w_in = ref.w.astype(np.complex64)
    ref.w = w_in.astype(np.complex128)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(beta=beta, drag=mu, viscosity=rate_for(nu_h, n, p), hyperP=p))
        load_state(s, w_in)
        set_fixed_dt(s, dt)
        s.setSplats([])
        s.encodeStep()
        ref.step(dt=dt)
        err1 = rel_l2(current_state(s), ref.w)
        assert err1 <= 1e-5, f"one step rel L2 {err1:.3e}"
        for _ in range(4):
            s.encodeStep()
            ref.step(dt=dt)
        err5 = rel_l2(current_state(s), ref.w)
        assert err5 <= 3e-5, f"five steps rel L2 {err5:.3e}"
    finally:
        s.destroy()


BIG_CASES = [
    # n, beta, mu, p, dt, amplitude -- the beta-plane configuration's coefficients at 4096^2
    # (hyperviscosity as the damping rate 1 at the cutoff)
    (2048, 0.0, 1e-2, 4, 1e-3, 8.0),
    (4096, 10.0, 5e-3, 4, 5e-4, 8.0),
]


@pytest.mark.parametrize("case", BIG_CASES, ids=[f"n{c[0]}" for c in BIG_CASES])
def test_fused_step_vs_oracle_large_grids(pkg, case):
    """One fused step at 2048^2 and 4096^2 (the 4096 tile shape: 2 columns per CTA)
    vs the FP64 oracle, rel L2 <= 1e-5."""
    n, beta, mu, p, dt, amp = case
    nu_h = 1.0 / (n / 3.0) ** (2 * p)
    ref = SpectralOracle(n=n, beta=beta, mu=mu, nu_h=nu_h, hyper_p=p)
    ref.set_vorticity(random_field(n, k0=n / 16, seed=n + 1, amplitude=amp))
    w_in = ref.w.astype(np.complex64)
    ref.w = w_in.astype(np.complex128)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(beta=beta, drag=mu, viscosity=rate_for(nu_h, n, p), hyperP=p))
        load_state(s, w_in)
        set_fixed_dt(s, dt)
        s.setSplats([])
        s.encodeStep()
        got = current_state(s)
    finally:
        s.destroy()
    ref.step(dt=dt)
    err = rel_l2(got, ref.w)
    print(f"n={n} one step rel L2 {err:.3e}")
    assert err <= 1e-5, f"one step rel L2 {err:.3e}"


def test_out_of_band_overflow_is_contained(pkg):
    """E(-dt/2) = exp(+205) beyond the dealias band overflows in FP32; the reference
    shader forms inf * 0 = NaN there (solver.wgsl:121).  Zero modes must stay zero and
    the step must match the FP64 oracle, whose factor does not overflow."""
    n, dt, rate = 256, 1e-3, 1000.0
    ref = SpectralOracle(n=n, nu_h=rate / (n / 3.0) ** 8, hyper_p=4)
    ref.set_vorticity(random_field(n, k0=20, seed=6, amplitude=4.0))
    w_in = ref.w.astype(np.complex64)
    ref.w = w_in.astype(np.complex128)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(viscosity=rate, hyperP=4))
        load_state(s, w_in)
        set_fixed_dt(s, dt)
        s.encodeStep()
        ref.step(dt=dt)
        got = current_state(s)
        assert np.all(np.isfinite(got))
        assert np.all(got[~dealias_mask(n)] == 0)
        assert rel_l2(got, ref.w) <= 1e-5
    finally:
        s.destroy()


def test_graph_replay_is_bitwise_identical(pkg):
    n = 256
    w = random_field(n, k0=20, seed=3, amplitude=4.0)
    outs = []
    for graph in (False, True):
        s = pkg.Solver.create(n=n, dyeScale=1)
        try:
            s.configure(config(viscosity=1.0, hyperP=4, forceAmp=0.1, forceK=30.0, forceWidth=2.0,
                               cfl=0.5, dtMax=2e-3))
            s.reset({"field": w, "dyePattern": "bands"})
            s.step(7, dye=True, reduce=True, graph=graph)
            outs.append((current_state(s), s.currentDye, s.getBuffer("dt")))
        finally:
            s.destroy()
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][2], outs[1][2])


# ---------------------------------------------------------------- Taylor-Green invariants
@pytest.mark.parametrize("n", [64, 256, 512])
def test_taylor_green_jacobian_vanishes(pkg, n):
    xs = np.arange(n) * 2 * np.pi / n
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    field = 6.0 * np.cos(2 * gx) * np.cos(2 * gy)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(viscosity=0.0, hyperP=1))
        s.seedPhysical(field)
        w = current_state(s)
        s.setBuffer("force", np.zeros((n, n), np.complex64))
        s.velocityPack(0)
        s.fft.inverse(None, "packA")
        s.fft.inverse(None, "packB")
        s.nlPack()
        s.fft.forward(None, "physZ")
        s.assemble()
        nl = np.max(np.abs(s.getBuffer("rhs"))) / np.max(np.abs(w))
        # FP32 round-off of the u*omega transforms (O(|omega| |u|) products, ~1e-7 per
        # pass, growing with log N) relative to the spectral amplitude of omega
        assert nl <= 1e-5, f"Jacobian/|w| = {nl:.3e}"
    finally:
        s.destroy()


@pytest.mark.parametrize("n", [64, 512])
def test_taylor_green_decay_rate(pkg, n):
    nu, dt, steps = 1e-3, 2e-3, 500
    xs = np.arange(n) * 2 * np.pi / n
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(viscosity=rate_for(nu, n, 1), hyperP=1))
        s.seedPhysical(6.0 * np.cos(2 * gx) * np.cos(2 * gy))
        w0 = current_state(s)[2, 2]
        set_fixed_dt(s, dt)
        for _ in range(steps):
            s.encodeStep()
        w1 = current_state(s)[2, 2]
        nu_h = s.paramsF[2]
        expected = np.exp(-float(nu_h) * 8.0 * dt * steps)
        assert abs(abs(w1 / w0) / expected - 1) <= 1e-5
    finally:
        s.destroy()


def test_inviscid_invariants(pkg):
    n, dt = 128, 2e-3
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(beta=12.0, viscosity=0.0, hyperP=4))
        s.seedPhysical(random_field(n, k0=10, seed=2))
        s.encodeDiagnostics(); s.copyDiagnostics()
        d0 = s.readDiagnostics()
        set_fixed_dt(s, dt)
        for _ in range(200):
            s.encodeStep()
        s.encodeDiagnostics(); s.copyDiagnostics()
        d1 = s.readDiagnostics()
        assert abs(d1["energy"] / d0["energy"] - 1) <= 2e-5
        assert abs(d1["enstrophy"] / d0["enstrophy"] - 1) <= 2e-5
    finally:
        s.destroy()


# ---------------------------------------------------------------- forcing
def test_stochastic_forcing_matches_restatement(pkg):
    n, dt = 128, 1e-3
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        for k in range(3):
            s.configure(config(forceAmp=0.1, forceK=20.0, forceWidth=2.0))
            set_fixed_dt(s, dt)
            s.setBuffer("physZ", np.zeros((n, n), np.complex64))
            s.setBuffer("force", np.zeros((n, n), np.complex64))
            s.assemble()
            want = wo.stochastic_forcing(n, 0.1, 20.0, 2.0, step_index=s.stepIndex, dt=dt)
            got = s.getBuffer("rhs")
            assert np.count_nonzero(want) > 0
            assert np.array_equal(got != 0, want != 0)
            assert rel_linf(got, want) <= 2e-6
            s.encodeStep()                      # advances stepIndex, latched at the next configure
    finally:
        s.destroy()


def test_stochastic_forcing_in_fused_step(pkg):
    n, dt = 128, 1e-3
    w = random_field(n, k0=12, seed=9, amplitude=3.0)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(viscosity=1.0, hyperP=4, forceAmp=0.1, forceK=24.0, forceWidth=2.0))
        s.seedPhysical(w)
        w_in = current_state(s)
        set_fixed_dt(s, dt)
        forcing = wo.stochastic_forcing(n, 0.1, 24.0, 2.0, step_index=0, dt=dt).astype(np.complex128)
        ref = SpectralOracle(n=n, nu_h=float(s.paramsF[2]), hyper_p=4)
        ref.w = w_in.astype(np.complex128)
        ref.step(dt=dt, forcing=forcing)
        s.encodeStep()
        assert rel_l2(current_state(s), ref.w) <= 1e-5
    finally:
        s.destroy()


def _splat(x, y, dx, dy, color=(1.0, 0.5, 0.25), radius=0.05, amp=400.0, dye=0.8):
    return {"x": x, "y": y, "dx": dx, "dy": dy, "color": color, "radius": radius, "amp": amp, "dyeAmp": dye}


def _splat_np(sp):
    r = np.zeros(1, wo.SPLAT_DTYPE)[0]
    r["x"], r["y"], r["dx"], r["dy"] = sp["x"], sp["y"], sp["dx"], sp["dy"]
    r["r"], r["g"], r["b"] = sp["color"]
    r["radius"], r["amp"], r["dye_amp"] = sp["radius"], sp["amp"], sp["dyeAmp"]
    return r


def test_pointer_force_spectrum(pkg):
    n = 128
    splats = [_splat(0.3, 0.6, 0.01, -0.02), _splat(0.95, 0.02, -0.015, 0.01, radius=0.08)]
    splats += [_splat(0.1 * i, 0.5, 0.01, 0.01) for i in range(1, 9)]     # 10 given, 8 used
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(viscosity=0.0))
        s.seedPhysical(np.zeros((n, n)))
        set_fixed_dt(s, 1e-3)
        s.setSplats(splats)
        s.encodeStep()
        got = s.getBuffer("force")
        want = np.fft.fft2(wo.pointer_force(n, [_splat_np(p) for p in splats[:8]]).astype(np.float64))
        assert rel_l2(got, want) <= 1e-5
        # with a zero initial state, one step equals the oracle step driven by that forcing
        ref = SpectralOracle(n=n)
        ref.step(dt=1e-3, forcing=want * dealias_mask(n))
        assert rel_l2(current_state(s), ref.w) <= 1e-5
    finally:
        s.destroy()


# ---------------------------------------------------------------- CFL reduction
def test_prime_cfl_dt(pkg):
    n = 256
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(cfl=0.5, dtMin=1e-5, dtMax=0.02))
        s.seedPhysical(random_field(n, k0=20, seed=4, amplitude=8.0))
        w = current_state(s)
        s.encodePrime()
        dt, speed = s.getBuffer("dt")[:2]
        ref = SpectralOracle(n=n, cfl=0.5, dt_max=0.02)
        ref.w = w.astype(np.complex128)
        u, v = ref.velocity()
        want_speed = np.max(np.abs(u) + np.abs(v))
        assert abs(speed / want_speed - 1) <= 2e-6
        want_dt, _ = wo.cfl_dt(u.astype(np.float32), v.astype(np.float32), n, 0.5, 1e-5, 0.02)
        assert abs(dt / want_dt - 1) <= 2e-6
        vel = s.getBuffer("vel")
        # u shares one complex transform with omega (two-for-one packing, solver.wgsl:38),
        # so its error is the transform's round-off scaled by |omega| / |u| (~16 here)
        assert rel_l2(vel.real + 0j, u) <= 5e-6 and rel_l2(vel.imag + 0j, v) <= 1e-6
    finally:
        s.destroy()


def test_adaptive_step_loop_reduces_each_substep(pkg):
    n = 128
    s = pkg.Solver.create(n=n, dyeScale=2)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMin=1e-5, dtMax=0.02))
        s.reset({"k0": 14, "amplitude": 6, "seed": 1})
        s.step(3, dye=True, reduce=True)
        vel = s.getBuffer("vel")
        want, _ = wo.cfl_dt(vel.real.astype(np.float32), vel.imag.astype(np.float32), n, 0.5, 1e-5, 0.02)
        # the same f32 operations on the same velocity: max(|u| + |v|), (cfl dx) / speed
        assert s.getBuffer("dt")[0] == want
        assert s.stepIndex == 3 and s.dyeParity == 1 and s.primed
    finally:
        s.destroy()


# ---------------------------------------------------------------- seeding
@pytest.mark.parametrize("n", [64, 256])
def test_fill_spectrum_seed(pkg, n):
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.seed(k0=14, amplitude=6, seed=1)
        got = s.getBuffer("state0")
        want = wo.fill_spectrum(n, 14, 6.0, 1)
        assert rel_linf(got, want) <= 1e-6
        assert np.array_equal(got != 0, want != 0)
        assert np.all(s.getBuffer("state1") == 0) and s.phase == 0
    finally:
        s.destroy()


def test_seed_physical_matches_set_vorticity(pkg):
    n = 128
    f = random_field(n, k0=10, seed=5, amplitude=3.0).astype(np.float32)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.seedPhysical(f)
        ref = SpectralOracle(n=n)
        ref.set_vorticity(f.astype(np.float64))
        assert rel_l2(s.getBuffer("state0"), ref.w) <= 1e-6
    finally:
        s.destroy()


def test_seed_band_statistics(pkg):
    n = 256
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.seedBand(6.0, 10.0, rms=1.0, seed=0)
        w = s.getBuffer("state0").astype(np.complex128)
        k = wavenumbers(n)
        kr = np.sqrt(k[None, :] ** 2 + k[:, None] ** 2)
        assert np.all(w[(kr < 6) | (kr > 10)] == 0)
        assert abs(np.sqrt(np.sum(np.abs(w) ** 2)) / (n * n) - 1.0) < 1e-5
        part = (-np.arange(n)) % n
        assert np.max(np.abs(w - np.conj(w[np.ix_(part, part)]))) == 0
        phys = np.fft.ifft2(w)
        assert abs(np.std(phys.real) - 1.0) < 1e-5
    finally:
        s.destroy()


@pytest.mark.parametrize("n,seed", [(256, 0), (1024, 1)])
def test_seed_band_matches_cpu_restatement(pkg, n, seed):
    """The benchmark's CPU arms start from wgsl_oracle.band_seed_spectrum: it must be the
    device seed's field (FP64 Box-Muller rounded to FP32 on both sides; libm and the
    FP64 sum order may differ in the last FP32 bit)."""
    from oracle.wgsl_oracle import band_seed_spectrum
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.seedBand(4.0, 12.0, rms=1.0, seed=seed)
        got = s.getBuffer("state0")
        want = band_seed_spectrum(n, 4.0, 12.0, 1.0, seed)
        assert np.array_equal(got != 0, want != 0)
        assert rel_l2(got, want) <= 1e-7
        assert np.max(np.abs(got - want)) <= 2e-7 * np.max(np.abs(want))
    finally:
        s.destroy()


@pytest.mark.parametrize("graph", [True, False])
def test_profiler_counts_every_kernel_class(pkg, graph):
    s = pkg.Solver.create(n=128, dyeScale=2)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMax=2e-3))
        s.reset({"k0": 14, "amplitude": 6, "seed": 1})
        s.profile(True)
        s.step(6, dye=True, reduce=True, graph=graph)
        s.profileRead()
        s.step(3, dye=True, reduce=True, graph=graph)
        p = s.profileRead()
        s.profile(False)
        assert p["phys_cols"][1] == 9 and p["spec_rows"][1] == 9 and p["dye"][1] == 3
        assert all(p[k][0] > 0 for k in ("phys_cols", "spec_rows", "dye"))
    finally:
        s.destroy()


# ---------------------------------------------------------------- tensor-core DFT-GEMM FFT
def test_tc_fft2_matches_numpy(pkg):
    """Split-FP16 tcgen05 DFT-GEMM 2D FFT at 1024^2 vs FP64 numpy (target rel L2 <= 1e-5)."""
    n = 1024
    rng = np.random.default_rng(7)
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    s = pkg.Solver.create(n=n, dyeScale=1, fft="tc-f16")
    try:
        s.setBuffer("packB", a)
        s.fft.forward(None, "packB")
        fwd = s.getBuffer("packB")
        err_f = rel_l2(fwd, np.fft.fft2(a.astype(np.complex128)))
        s.fft.inverse(None, "packB")
        err_rt = rel_l2(s.getBuffer("packB"), a)
        s.setBuffer("packB", a)
        s.fft.inverse(None, "packB")
        err_i = rel_l2(s.getBuffer("packB"), np.fft.ifft2(a.astype(np.complex128)))
        print(f"tc fft2 rel L2: forward {err_f:.3e} inverse {err_i:.3e} round trip {err_rt:.3e}")
        assert err_f <= 1e-5 and err_i <= 1e-5 and err_rt <= 2e-5
    finally:
        s.destroy()


def test_tc_precision_sizes(pkg):
    """The tensor-core FFT exists at 256, 512, 1024, 2048 and 4096; smaller grids are
    refused with S2D_ERR_UNSUPPORTED_N."""
    for fft in ("tc-f16", "tc-bf16"):
        for n in (32, 64, 128):
            with pytest.raises(pkg.S2DError) as ei:
                pkg.Solver.create(n=n, fft=fft)
            assert ei.value.status == -2


@pytest.mark.parametrize("n", [256, 512, 2048, 4096])
@pytest.mark.parametrize("fft", ["tc-f16", "tc-bf16"])
def test_tc_generic_fft2_matches_numpy(pkg, n, fft):
    """The N1 x N2 tensor-core 2D transforms (the grid sizes other than 1024), forward
    unscaled and inverse scaled 1/N per pass (fft.js:58-59), against numpy in FP64."""
    rng = np.random.default_rng(n)
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    s = pkg.Solver.create(n=n, dyeScale=1, fft=fft)
    try:
        s.setBuffer("packB", a)
        s.fft.forward(None, "packB")
        e_fwd = rel_l2(s.getBuffer("packB"), np.fft.fft2(a.astype(np.complex128)))
        s.setBuffer("packB", a)
        s.fft.inverse(None, "packB")
        e_inv = rel_l2(s.getBuffer("packB"), np.fft.ifft2(a.astype(np.complex128)))
        s.synchronize()
    finally:
        s.destroy()
    print(f"{fft} {n}^2 2D FFT rel L2: forward {e_fwd:.3e} inverse {e_inv:.3e}")
    bound = 5e-6 if fft == "tc-f16" else 2e-5
    assert e_fwd <= bound and e_inv <= bound


@pytest.mark.parametrize("fft", ["tc-f16", "tc-bf16"])
@pytest.mark.parametrize("n", [512, 1024])
def test_tc_localised_field_stays_finite(pkg, n, fft):
    """A localised field (a Gaussian vortex whose far-field rows underflow to zero or to
    subnormal values) through the tensor-core transforms: the per-row power-of-two scales
    stay finite, and the step matches the FP64 oracle."""
    xs = np.arange(n) * 2 * np.pi / n
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    field = np.exp(-((gx - np.pi) ** 2 + (gy - np.pi) ** 2) / 0.22 ** 2)
    dt = 5e-3
    s = pkg.Solver.create(n=n, dyeScale=1, fft=fft)
    try:
        s.configure(config(viscosity=0.0, hyperP=1))
        s.seedPhysical(field)
        w0 = current_state(s)
        assert np.all(np.isfinite(w0))
        ref = SpectralOracle(n=n)
        ref.set_vorticity(field)
        assert rel_l2(w0, ref.w) <= 2e-5
        ref.w = w0.astype(np.complex128)
        set_fixed_dt(s, dt)
        s.encodeStep()
        ref.step(dt=dt)
        got = current_state(s)
        s.synchronize()
    finally:
        s.destroy()
    assert np.all(np.isfinite(got))
    assert rel_l2(got, ref.w) <= 2e-5


@pytest.mark.parametrize("n", [256, 512, 2048])
@pytest.mark.parametrize("fft", ["tc-f16", "tc-bf16"])
def test_tc_unfused_step_vs_oracle(pkg, n, fft):
    """Tensor-core solvers at the sizes without fused tensor-core stages run the reference's
    per-stage order with every 2D transform on the tensor cores: rel L2 to the FP64 oracle
    <= 1e-5 after one step (beta, hyperviscosity, drag), <= 3e-5 after three."""
    mu, p, dt, beta = 1e-2, 4, 1e-3, 10.0
    nu_h = 1.0 / (n / 3.0) ** 8
    ref = SpectralOracle(n=n, beta=beta, mu=mu, nu_h=nu_h, hyper_p=p)
    ref.set_vorticity(random_field(n, k0=n / 16, seed=13, amplitude=8.0))
    w_in = ref.w.astype(np.complex64)
    ref.w = w_in.astype(np.complex128)
    s = _tc_case_solver(pkg, fft, n, beta, mu, nu_h, p, w_in, dt)
    try:
        s.encodeStep()
        ref.step(dt=dt)
        err1 = rel_l2(current_state(s), ref.w)
        for _ in range(2):
            s.encodeStep()
            ref.step(dt=dt)
        err3 = rel_l2(current_state(s), ref.w)
        s.synchronize()
    finally:
        s.destroy()
    print(f"{fft} {n}^2 unfused tensor-core step rel L2: 1 step {err1:.3e}, 3 steps {err3:.3e}")
    assert err1 <= 1e-5 and err3 <= 3e-5


def test_precision_sweep_fft_and_step(pkg):
    """FP32, FP16-split and BF16-split FFT paths at 1024^2 against FP64: 2D FFT and one
    fused step (rel L2, printed).  FP32 and the FP16 split meet 1e-5; the BF16 split keeps
    16 significant bits per operand (the FP16 split 22), so its error is larger but still
    under the 1e-5 bar."""
    n, dt = 1024, 1e-3
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    fa = np.fft.fft2(a.astype(np.complex128))
    nu_h = 1.0 / (n / 3.0) ** 8
    ref = SpectralOracle(n=n, beta=10.0, mu=1e-2, nu_h=nu_h, hyper_p=4)
    ref.set_vorticity(random_field(n, k0=n / 8, seed=21, amplitude=8.0))
    w_in = ref.w.astype(np.complex64)
    ref.w = w_in.astype(np.complex128)
    ref.step(dt=dt)
    errs = {}
    for fft in ("fp32", "tc-f16", "tc-bf16"):
        s = pkg.Solver.create(n=n, dyeScale=1, fft=fft)
        try:
            s.setBuffer("packB", a)
            s.fft.forward(None, "packB")
            e_fft = rel_l2(s.getBuffer("packB"), fa)
            s.configure(config(beta=10.0, drag=1e-2, viscosity=rate_for(nu_h, n, 4), hyperP=4))
            load_state(s, w_in)
            set_fixed_dt(s, dt)
            s.setSplats([])
            s.encodeStep()
            e_step = rel_l2(current_state(s), ref.w)
        finally:
            s.destroy()
        errs[fft] = (e_fft, e_step)
        print(f"{fft}: 2D FFT rel L2 {e_fft:.3e}, one step rel L2 {e_step:.3e}")
    assert errs["fp32"][0] <= 1e-5 and errs["fp32"][1] <= 1e-5
    assert errs["tc-f16"][0] <= 1e-5 and errs["tc-f16"][1] <= 1e-5
    # the BF16 split keeps 16 significant bits per operand (6.5e-6 / 2.5e-6 measured): it
    # meets the same 1e-5 bar with less margin than the FP16 split
    assert errs["tc-bf16"][0] <= 1e-5 and errs["tc-bf16"][1] <= 1e-5
    assert errs["tc-bf16"][0] > errs["tc-f16"][0]


def _tc_rows(s):
    """Pin the row stage of tensor-core solver `s` to the tensor-core row kernel."""
    names = s.tuneVariantNames("row")
    assert names[-1].startswith("tensor-core rows")
    s.tuneSelect(0, len(names) - 1)


def _tc_case_solver(pkg, fft, n, beta, mu, nu_h, p, w_in, dt, rows="fp32"):
    s = pkg.Solver.create(n=n, dyeScale=1, fft=fft)
    if rows == "tc":
        _tc_rows(s)
    s.configure(config(beta=beta, drag=mu, viscosity=rate_for(nu_h, n, p), hyperP=p))
    load_state(s, w_in)
    set_fixed_dt(s, dt)
    s.setSplats([])
    return s


@pytest.mark.parametrize("rows", ["fp32", "tc"])
@pytest.mark.parametrize("fft", ["tc-f16", "tc-bf16"])
@pytest.mark.parametrize("beta", [0.0, 10.0])
def test_tc_fused_step_vs_oracle(pkg, beta, fft, rows):
    """Fused RK3 step with the tensor-core column stage (split FP16 / BF16 DFT-GEMMs),
    with the FP32 or the tensor-core row stage, vs the FP64 oracle at 1024^2: rel L2
    <= 1e-5 after one step, <= 3e-5 after five."""
    n, mu, p, dt, amp = 1024, 1e-2, 4, 1e-3, 8.0
    nu_h = 1.0 / (n / 3.0) ** 8
    ref = SpectralOracle(n=n, beta=beta, mu=mu, nu_h=nu_h, hyper_p=p)
    ref.set_vorticity(random_field(n, k0=n / 8, seed=11, amplitude=amp))
    w_in = ref.w.astype(np.complex64)
    ref.w = w_in.astype(np.complex128)
    s = _tc_case_solver(pkg, fft, n, beta, mu, nu_h, p, w_in, dt, rows=rows)
    try:
        s.encodeStep()
        ref.step(dt=dt)
        err1 = rel_l2(current_state(s), ref.w)
        for _ in range(4):
            s.encodeStep()
            ref.step(dt=dt)
        err5 = rel_l2(current_state(s), ref.w)
        print(f"{fft} rows={rows} fused step rel L2: 1 step {err1:.3e}, 5 steps {err5:.3e}")
        assert err1 <= 1e-5, f"one step rel L2 {err1:.3e}"
        assert err5 <= 3e-5, f"five steps rel L2 {err5:.3e}"
    finally:
        s.destroy()


def test_tc_prime_velocity_and_dt(pkg):
    """encodePrime through the tensor-core column stage: velocity vs the FP32 path and
    the CFL dt from its max |u|+|v|."""
    n = 1024
    w = random_field(n, k0=40, seed=5, amplitude=6.0)
    out = {}
    for fft in ("fp32", "tc-f16"):
        s = pkg.Solver.create(n=n, dyeScale=1, fft=fft)
        try:
            s.configure(config(viscosity=1.0, cfl=0.5, dtMax=1.0))
            s.seedPhysical(w)
            s.encodePrime()
            out[fft] = (s.getBuffer("vel"), s.getBuffer("dt"))
        finally:
            s.destroy()
    v32, d32 = out["fp32"]
    vtc, dtc = out["tc-f16"]
    assert rel_l2(vtc, v32) <= 1e-5
    assert abs(float(dtc[1]) / float(d32[1]) - 1) <= 1e-5
    assert abs(float(dtc[0]) / float(d32[0]) - 1) <= 1e-5


def test_tc_forced_run_tracks_fp32(pkg):
    """Forced, adaptive-dt run with dye (the 1024^2 benchmark configuration) through the
    tensor-core column stage stays within 1e-5 (rel L2) of the FP32 path after 5 steps,
    and the dt chain agrees."""
    n = 1024
    w = random_field(n, k0=14, seed=1, amplitude=6.0)
    out = {}
    for key in ("fp32", "tc-f16", "tc-f16+rows"):
        s = pkg.Solver.create(n=n, dyeScale=1, fft=key.split("+")[0])
        try:
            if key.endswith("+rows"):
                _tc_rows(s)
            s.configure(config(viscosity=1.0, hyperP=4, drag=1e-2, forceAmp=0.1, forceK=64.0, forceWidth=2.0,
                               cfl=0.5, dtMax=1e-3))
            s.reset({"field": w, "dyePattern": "bands"})
            s.setSplats([{"x": 0.3, "y": 0.6, "dx": 2.0, "dy": -1.0, "color": [1.0, 0.5, 0.2], "radius": 0.03,
                          "amp": 1.0, "dyeAmp": 1.0}])
            s.step(5, dye=True, reduce=True, graph=True)
            out[key] = (current_state(s), s.getBuffer("dt"), s.getBuffer("vel"))
        finally:
            s.destroy()
    for key in ("tc-f16", "tc-f16+rows"):
        e_state = rel_l2(out[key][0], out["fp32"][0])
        e_vel = rel_l2(out[key][2], out["fp32"][2])
        print(f"{key} vs fp32 after 5 forced steps (stochastic + pointer forcing): state {e_state:.3e} vel {e_vel:.3e}")
        assert e_state <= 1e-5 and e_vel <= 1e-5
        assert abs(float(out[key][1][0]) / float(out["fp32"][1][0]) - 1) <= 1e-5


@pytest.mark.parametrize("rows", ["fp32", "tc"])
def test_tc_taylor_green_decay_rate(pkg, rows):
    """Taylor-Green through the tensor-core step at 1024^2: the (2,2) mode decays as
    exp(-nu |k|^2 t) to 1e-5 (the Jacobian error of the split-FP16 transforms feeds
    straight into that mode)."""
    n, nu, dt, steps = 1024, 1e-3, 2e-3, 200
    xs = np.arange(n) * 2 * np.pi / n
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    s = pkg.Solver.create(n=n, dyeScale=1, fft="tc-f16")
    if rows == "tc":
        _tc_rows(s)
    try:
        s.configure(config(viscosity=rate_for(nu, n, 1), hyperP=1))
        s.seedPhysical(6.0 * np.cos(2 * gx) * np.cos(2 * gy))
        w0 = current_state(s)[2, 2]
        set_fixed_dt(s, dt)
        for _ in range(steps):
            s.encodeStep()
        w1 = current_state(s)[2, 2]
        nu_h = s.paramsF[2]
        expected = np.exp(-float(nu_h) * 8.0 * dt * steps)
        err = abs(abs(w1 / w0) / expected - 1)
        print(f"tc rows={rows} Taylor-Green decay-rate error {err:.3e}")
        assert err <= 1e-5
    finally:
        s.destroy()


def test_relatch_equals_configure_per_substep(pkg):
    """S2D_STEP_RELATCH (stepIndex latched by the step's first column kernel) draws the
    same forcing phases as a configure() before every substep (solver.js:316), directly
    and through graph replay."""
    n = 128
    w = random_field(n, k0=12, seed=9, amplitude=4.0)
    cfg = config(viscosity=1.0, hyperP=4, forceAmp=0.1, forceK=20.0, forceWidth=2.0, cfl=0.5, dtMax=2e-3)
    outs = []
    for mode in ("configure", "relatch", "relatch-graph"):
        s = pkg.Solver.create(n=n, dyeScale=1)
        try:
            s.configure(cfg)
            s.reset({"field": w, "dyePattern": "none"})
            for _ in range(4):
                if mode == "configure":
                    s.configure(cfg)
                    s.step(1, dye=False, reduce=True, graph=False)
                else:
                    s.step(1, dye=False, reduce=True, graph=(mode == "relatch-graph"), relatch=True)
            outs.append(current_state(s))
        finally:
            s.destroy()
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], outs[2])


def test_skipped_zero_rows_read_back_as_zero(pkg):
    """The row kernel leaves pack rows that are entirely zero unwritten (and flags them for
    the column kernels); any other reader sees them as zeros.  Garbage written into the
    packs beforehand must not survive into getBuffer or into the step."""
    n = 256
    ref = SpectralOracle(n=n, nu_h=1.0 / (n / 3.0) ** 8, hyper_p=4)
    ref.set_vorticity(random_field(n, k0=20, seed=4, amplitude=5.0))       # dealiased
    w_in = ref.w.astype(np.complex64)
    ref.w = w_in.astype(np.complex128)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(viscosity=1.0, hyperP=4))
        rng = np.random.default_rng(1)
        junk = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
        s.setBuffer("packA", junk)
        s.setBuffer("packB", junk)
        load_state(s, w_in)
        set_fixed_dt(s, 1e-3)
        s.encodeStep()
        ref.step(dt=1e-3)
        assert rel_l2(current_state(s), ref.w) <= 1e-5
        ky = np.fft.fftfreq(n, 1.0 / n)
        out_rows = np.abs(ky) >= n / 3.0
        for name in ("packA", "packB"):
            p = s.getBuffer(name)
            assert np.all(p[out_rows] == 0), name
            assert np.any(p[~out_rows] != 0), name
    finally:
        s.destroy()
