"""Diagnostics (FP64 and the reference's fixed point) and dye advection."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_helpers import config, current_state, set_fixed_dt
from oracle import wgsl_oracle as wo
from oracle.spectral_oracle import SpectralOracle, random_field

pytestmark = pytest.mark.gpu


def test_read_before_copy_is_null(pkg):
    s = pkg.Solver.create(n=64, dyeScale=1)
    try:
        assert s.readDiagnostics() is None                                  # solver.js:571-573
        s.encodeDiagnostics()
        s.copyDiagnostics()
        assert s.readDiagnostics() is not None
        assert s.readDiagnostics() is None                                  # read state back to idle
    finally:
        s.destroy()


def _same_diagnostics(a, b, what):
    """Diagnostics of one state: the zonal mean bit for bit, the FP64 sums (added across
    CTAs in any order) to their rounding."""
    assert np.array_equal(a["zonal"], b["zonal"]), what
    assert np.allclose(a["spectrum"], b["spectrum"], rtol=1e-13, atol=1e-300), what
    for key in ("energy", "enstrophy"):
        assert abs(a[key] - b[key]) <= 1e-13 * abs(b[key]), (what, key)


def _diag_after_steps(pkg, n, steps, graph, between):
    """Diagnostics of the state after `steps` steps, with `between(s)` run between
    encodeDiagnostics and copyDiagnostics; returns the read result and the dt slots read
    after it."""
    s = pkg.Solver.create(n=n, dyeScale=2)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMax=0.01))
        s.seedPhysical(random_field(n, k0=n / 10, seed=11, amplitude=5.0))
        for _ in range(steps):
            s.step(1, dye=True, reduce=True, graph=graph)
        s.encodeDiagnostics()
        between(s)
        s.copyDiagnostics()
        d = s.readDiagnostics()
        return d, s.getBuffer("dt")[:2].copy()
    finally:
        s.destroy()


@pytest.mark.parametrize("graph", [False, True])
def test_diagnostics_run_alongside_the_next_steps(pkg, graph):
    """The spectra run on a second stream alongside the next step, and the calls after them
    are ordered so that the result is the state at encodeDiagnostics: steps (one, then a
    second that rewrites the state buffer the spectra read), a reseed, a second encode and
    multi-substep calls leave it unchanged (the zonal mean bit for bit, the FP64 sums to
    their rounding: CTAs add them in any order; a spectrum of a later state would differ in
    the third digit); dt is the slot current at the copy (solver.js:560-568)."""
    n = 256
    base, _ = _diag_after_steps(pkg, n, 3, graph, lambda s: None)
    cases = {
        "one step": lambda s: s.step(1, dye=True, reduce=True, graph=graph),
        "three steps": lambda s: [s.step(1, dye=True, reduce=True, graph=graph) for _ in range(3)],
        "substeps": lambda s: s.step(4, dye=True, reduce=True, graph=graph),
        "reseed": lambda s: s.seed(k0=9, amplitude=3, seed=5),
        # a phase moved back one place makes the next step write the buffer just read
        "phase moved": lambda s: (setattr(s, "phase", (s.phase + 2) % 3),
                                  s.step(1, dye=True, reduce=True, graph=graph)),
    }
    for name, between in cases.items():
        d, dt_now = _diag_after_steps(pkg, n, 3, graph, between)
        _same_diagnostics(d, base, name)
        assert d["dt"] == dt_now[0] and d["maxSpeed"] == dt_now[1], name

    # a second encode before the copy: the copy reads the later block, equal to the
    # diagnostics of the same state encoded once
    def twice(s):
        s.step(1, dye=True, reduce=True, graph=graph)
        s.encodeDiagnostics()
    d2, _ = _diag_after_steps(pkg, n, 3, graph, twice)
    once, _ = _diag_after_steps(pkg, n, 4, graph, lambda s: None)
    _same_diagnostics(d2, once, "second encode")


def test_diagnostics_captured_by_the_caller(pkg):
    """encodeDiagnostics captured into a caller's graph on the solver's stream (the spectra
    then stay on that stream, and the graph clears the block it fills): replayed three
    times, it gives the diagnostics of the state, as a plain call does."""
    import torch
    n = 128
    s = pkg.Solver.create(n=n, dyeScale=2)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMax=0.01))
        s.seedPhysical(random_field(n, k0=12, seed=6, amplitude=5.0))
        s.step(2, dye=True, reduce=True, graph=True)
        s.encodeDiagnostics(); s.copyDiagnostics()
        ref = s.readDiagnostics()
        s.synchronize()
        st = torch.cuda.ExternalStream(s.stream)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=st):
            s.encodeDiagnostics()
        with torch.cuda.stream(st):   # replayed on the solver's stream, in its order
            for _ in range(3):
                g.replay()
        torch.cuda.synchronize()
        s.copyDiagnostics()
        _same_diagnostics(s.readDiagnostics(), ref, "captured")
        del g
    finally:
        s.destroy()


def test_pipelined_readback_matches_synchronous(pkg):
    """The frame-loop order of the end-to-end benchmark (step k, encode k, read k-1,
    copy k) gives, for every step, the diagnostics a synchronous encode-copy-read of the
    same state gives."""
    n, steps = 128, 6
    sync = []
    s = pkg.Solver.create(n=n, dyeScale=2)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMax=0.01))
        s.seedPhysical(random_field(n, k0=12, seed=4, amplitude=5.0))
        for _ in range(steps):
            s.step(1, dye=True, reduce=True, graph=True)
            s.encodeDiagnostics(); s.copyDiagnostics()
            sync.append(s.readDiagnostics())
    finally:
        s.destroy()
    piped = []
    s = pkg.Solver.create(n=n, dyeScale=2)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMax=0.01))
        s.seedPhysical(random_field(n, k0=12, seed=4, amplitude=5.0))
        for _ in range(steps):
            s.step(1, dye=True, reduce=True, graph=True)
            s.encodeDiagnostics()
            d = s.readDiagnostics()
            if d is not None:
                piped.append(d)
            s.copyDiagnostics()
        piped.append(s.readDiagnostics())
    finally:
        s.destroy()
    assert len(piped) == steps
    for k, (a, b) in enumerate(zip(sync, piped)):
        _same_diagnostics(a, b, k)
        assert a["dt"] == b["dt"] and a["maxSpeed"] == b["maxSpeed"], k


@pytest.mark.parametrize("n", [32, 64, 512, 2048])
def test_fp64_diagnostics(pkg, n):
    """Every k-space tile geometry of the diagnostics kernel: a tile spanning the whole
    grid (32), whole rows of both signs (64), and 64 x 32 tiles of one sign (512, 2048)."""
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMax=0.01))
        s.seedPhysical(random_field(n, k0=n / 10, seed=7, amplitude=5.0))
        s.encodePrime()
        w = current_state(s)
        s.encodeDiagnostics()
        s.copyDiagnostics()
        d = s.readDiagnostics()
        ref = SpectralOracle(n=n)
        ref.w = w.astype(np.complex128)
        assert abs(d["energy"] / ref.energy() - 1) <= 1e-12
        assert abs(d["enstrophy"] / ref.enstrophy() - 1) <= 1e-12
        assert np.allclose(d["spectrum"], ref.spectrum()[1], rtol=1e-11, atol=1e-300)
        # zonal mean of u of the last velocity evaluation (here: the prime's, from w)
        zonal_ref = ref.zonal_mean_u()
        assert np.max(np.abs(d["zonal"] - zonal_ref)) <= 1e-5 * np.max(np.abs(ref.velocity()[0]))
        dt, speed = s.getBuffer("dt")[:2]
        assert d["dt"] == dt and d["maxSpeed"] == speed
    finally:
        s.destroy()


def test_zonal_mean_is_the_stage2_velocity(pkg):
    n, dt = 128, 2e-3
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(beta=10.0, viscosity=1.0))
        s.seedPhysical(random_field(n, k0=12, seed=8, amplitude=6.0))
        w0 = current_state(s)
        set_fixed_dt(s, dt)
        s.encodeStep()
        s.encodeDiagnostics(); s.copyDiagnostics()
        d = s.readDiagnostics()
        ref = SpectralOracle(n=n, beta=10.0, nu_h=float(s.paramsF[2]), hyper_p=4)
        w = w0.astype(np.complex128)
        e_full, e_half, e_mh = ref.factor(dt), ref.factor(dt / 2), ref.factor(-dt / 2)
        w1 = e_full * (w + dt * ref.rhs(w))
        w2 = 0.75 * e_half * w + 0.25 * e_mh * (w1 + dt * ref.rhs(w1))
        ref.w = w2                          # the reference reads packA.y after stage 2 (solver.js:258)
        want = ref.zonal_mean_u()
        assert np.max(np.abs(d["zonal"] - want)) <= 2e-5 * np.max(np.abs(ref.velocity()[0]))
    finally:
        s.destroy()


@pytest.mark.parametrize("n", [32, 128, 1024])
def test_fixed_point_diagnostics_match_restatement(pkg, n):
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.seed(k0=14, amplitude=6, seed=3)
        s.encodeDiagnostics(); s.copyDiagnostics()
        s.readDiagnostics()
        fx = s.readDiagnosticsFixed()
        spec, e, z = wo.spectrum_fixed_point(s.getBuffer("state0"), n)
        # integer sums of the same f32 per-cell values (squares rounded before their sum,
        # correctly rounded quotient and square root): equal u32 counters, so equal decodes
        assert np.array_equal(fx["spectrum"], spec.astype(np.float32))
        assert fx["energy"] == float(np.float32(e)) and fx["enstrophy"] == float(np.float32(z))
    finally:
        s.destroy()


# ---------------------------------------------------------------- dye
@pytest.mark.parametrize("m_scale", [1, 2])
def test_paint_bands(pkg, m_scale):
    n = 64
    s = pkg.Solver.create(n=n, dyeScale=m_scale)
    try:
        s.reset({"k0": 14, "amplitude": 6, "seed": 1, "dyePattern": "bands"})
        got = s.currentDye
        want = wo.paint_dye_bands(n * m_scale)
        # toHalf (solver.js:20-41) is integer work on the FP32 rounding of the same double
        # expression: bit for bit
        diff = np.abs(got.astype(np.int32) - want.astype(np.int32))
        assert np.count_nonzero(diff) == 0, f"{np.count_nonzero(diff)} texel channels differ, max {diff.max()}"
    finally:
        s.destroy()


def _splat_np(sp):
    r = np.zeros(1, wo.SPLAT_DTYPE)[0]
    r["x"], r["y"], r["dx"], r["dy"] = sp["x"], sp["y"], sp["dx"], sp["dy"]
    r["r"], r["g"], r["b"] = sp["color"]
    r["radius"], r["amp"], r["dye_amp"] = sp["radius"], sp["amp"], sp["dyeAmp"]
    return r


@pytest.mark.parametrize("m_scale", [1, 2, 4])
def test_dye_bfecc_step(pkg, m_scale):
    n = 128
    s = pkg.Solver.create(n=n, dyeScale=m_scale)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMax=0.02, dyeFade=0.999))
        s.reset({"k0": 10, "amplitude": 8, "seed": 2, "dyePattern": "bands"})
        splat = {"x": 0.4, "y": 0.7, "dx": 0.01, "dy": 0.0, "color": (1.0, 0.42, 0.28), "radius": 0.05,
                 "amp": 0.0, "dyeAmp": 0.9}
        s.setSplats([splat])
        s.encodePrime()
        dye0 = s.currentDye
        vel = s.getBuffer("vel")
        dt = float(s.getBuffer("dt")[0])
        s.encodeDye()
        got = wo.half_bits_to_f32(s.currentDye)
        velf = np.stack([vel.real, vel.imag], axis=-1).astype(np.float32)
        want_bits = wo.dye_step(dye0, velf, dt, 0.999, [_splat_np(splat)])
        want = wo.half_bits_to_f32(want_bits)
        # the restatement evaluates the kernels' FP32 operations in the same order with the
        # same fused multiply-adds: texels untouched by the splat are bit-exact.  Inside the
        # splat the weight uses expf, whose CUDA and NumPy results may differ in the last
        # FP32 bit: one unit in the last place, on at most 1 % of the channels.
        px = (np.arange(n * m_scale) + 0.5) / (n * m_scale)
        rx = (px[None, :] - splat["x"] + 0.5) % 1.0 - 0.5
        ry = (px[:, None] - splat["y"] + 0.5) % 1.0 - 0.5
        near = (rx * rx + ry * ry) < 9.0 * splat["radius"] ** 2 * 1.01
        gb = s.currentDye.astype(np.int32)
        wb = want_bits.astype(np.int32)
        far = ~near
        assert np.array_equal(gb[far], wb[far]), int(np.count_nonzero(gb[far] != wb[far]))
        assert np.max(np.abs(gb[near] - wb[near])) <= 1
        assert np.mean(gb[near] != wb[near]) <= 1e-2
        assert np.all(got[..., 3] == 1.0)
    finally:
        s.destroy()


@pytest.mark.parametrize("n,m_scale", [(64, 1), (128, 2), (256, 4)])
def test_fused_dye_equals_three_passes(pkg, n, m_scale):
    """The one-launch dye step reproduces the reference's three dispatches bit for bit:
    at the CFL dt (tiles whose traces stay under one texel take the untested window
    lookups), at a dt moving the fastest traces 1.5 texels (tiles of both kinds in one
    launch) and at a dt moving them several texels (back-traces past the on-chip halo,
    recomputed from global memory)."""
    splat = {"x": 0.1, "y": 0.9, "dx": -0.01, "dy": 0.02, "color": (0.36, 0.93, 0.66), "radius": 0.08,
             "amp": 0.0, "dyeAmp": 1.0}
    outs = []
    for fused in (True, False):
        s = pkg.Solver.create(n=n, dyeScale=m_scale)
        try:
            s.configure(config(viscosity=1.0, cfl=0.5, dtMax=0.02, dyeFade=0.99))
            s.reset({"k0": 8, "amplitude": 10, "seed": 4, "dyePattern": "bands"})
            s.setSplats([splat])
            s.encodePrime()
            vel = s.getBuffer("vel")
            vmax = float(max(np.abs(vel.real).max(), np.abs(vel.imag).max()))
            dt_mixed = 1.5 * 2 * np.pi / (vmax * n * m_scale)
            for dt in (None, dt_mixed, 0.05):
                if dt is not None:
                    set_fixed_dt(s, dt)
                for _ in range(2):
                    (s.encodeDye if fused else s.encodeDyePasses)()
                outs.append(s.currentDye)
        finally:
            s.destroy()
    assert np.array_equal(outs[0], outs[3])
    assert np.array_equal(outs[1], outs[4])
    assert np.array_equal(outs[2], outs[5])
