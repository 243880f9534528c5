"""C-ABI library and host-logic checks that need no GPU (no compute calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle import fft_oracle as fo
from oracle import wgsl_oracle as wo

HEADER = os.path.join(ROOT, "include", "s2d.h")


def _declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(s2d_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol(pkg):
    lib = pkg.lib()
    declared = _declared_symbols()
    assert len(declared) > 40
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    from importlib import import_module
    protos = import_module(pkg.__name__ + "._lib").PROTOTYPES
    assert sorted(protos) == declared      # the ctypes binding covers exactly the header


def test_library_is_sm100a_only():
    so = os.path.join(ROOT, "spectral-2d-turbulence_b200", "libs2d.so")
    data = open(so, "rb").read()
    assert b"sm_100a" in data


def test_status_strings(pkg):
    lib = pkg.lib()
    assert lib.s2d_version() >= 10000
    for st in (0, 1, -1, -2, -3, -4, -5, -6, -7):
        assert lib.s2d_status_string(st)


@pytest.mark.parametrize("n", [2, 8, 32, 128, 512, 2048, 4, 16, 64, 256, 1024, 4096])
def test_radix_schedule_matches_reference(pkg, n):
    r = pkg.radixSchedule(n)
    rad = fo.radix_schedule(n)
    assert r["stages"] == rad.count(4)
    assert r["hasRadix2"] == (2 in rad)


@pytest.mark.parametrize("n", [3, 12, 48, 100])
def test_radix_schedule_throws(pkg, n):
    with pytest.raises(pkg.S2DError) as ei:
        pkg.radixSchedule(n)
    assert ei.value.status == -2


def test_create_without_gpu_fails_loudly(pkg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(pkg.S2DError) as ei:
        pkg.Solver.create(n=64, dyeScale=1)
    assert ei.value.status in (-7, -3)


def test_unknown_fft_arithmetic_rejected(pkg):
    with pytest.raises(ValueError):
        pkg.Solver.create(n=64, fft="fp8")


@pytest.mark.parametrize("scale", [0, 3, 5, 8])
def test_dye_scale_must_be_a_power_of_two(pkg, scale):
    """The dye grid wraps texel indices with a power-of-two mask: dyeScale 1, 2 (the
    reference's choices, main.js:196) or 4; the check precedes any device work."""
    with pytest.raises(pkg.S2DError) as ei:
        pkg.Solver.create(n=64, dyeScale=scale)
    assert ei.value.status == -1


# ---------------------------------------------------------------- WGSL restatement self-checks
def test_hash_matches_js_imul_semantics():
    # hash32 (solver.js:43-47) written with JS-style 32-bit wrapping in Python ints
    def js_hash(x):
        v = ((x & 0xFFFFFFFF) * 747796405 + 2891336453) & 0xFFFFFFFF
        v = (((v >> ((v >> 28) + 4)) ^ v) * 277803737) & 0xFFFFFFFF
        return ((v >> 22) ^ v) & 0xFFFFFFFF
    xs = np.array([0, 1, 2, 12345, 0xFFFFFFFF, 0x80000000, 747796405], np.uint32)
    assert [int(h) for h in wo.hash1(xs)] == [js_hash(int(x)) for x in xs]


def test_stochastic_forcing_is_hermitian_and_annular():
    n = 64
    f = wo.stochastic_forcing(n, force_amp=0.1, force_k=12.0, force_width=2.0, step_index=7, dt=1e-3)
    part = (-np.arange(n)) % n
    mirror = np.conj(f[np.ix_(part, part)])
    assert np.max(np.abs(f - mirror)) <= 1e-6 * np.max(np.abs(f))
    k = wo.wn_f32(n).astype(np.float64)
    kr = np.sqrt(k[None, :] ** 2 + k[:, None] ** 2)
    on = np.abs(f) > 0
    assert on.any()
    assert np.all(np.abs(kr[on] - 12.0) <= 2.0 * np.sqrt(np.log(1e4)) + 1e-6)


def test_fill_spectrum_rms_and_hermitian():
    n = 64
    d = wo.fill_spectrum(n, k0=14, amplitude=6.0, seed=1).astype(np.complex128)
    rms = np.sqrt(np.sum(np.abs(d) ** 2)) / (n * n)
    assert abs(rms / 6.0 - 1) < 1e-5
    part = (-np.arange(n)) % n
    assert np.max(np.abs(d - np.conj(d[np.ix_(part, part)]))) < 1e-5 * np.max(np.abs(d))
    phys = np.fft.ifft2(d)
    assert np.max(np.abs(phys.imag)) < 1e-6 * np.max(np.abs(phys.real))


def test_to_half_truncates():
    vals = np.array([1.0, 0.5, 0.1, 0.3333333, 65504.0, 1e-6, 7e-5, -2.5], np.float32)
    bits = wo.to_half_bits(vals)
    back = wo.half_bits_to_f32(bits)
    assert np.all(np.abs(back) <= np.abs(vals) + 1e-12)       # truncation toward zero
    assert np.all(np.abs(back - vals) <= np.abs(vals) * 2 ** -10 + 6e-8)
    assert int(wo.to_half_bits(np.float32(1.0))) == 0x3C00


def test_pointer_force_is_a_curl():
    n = 64
    sp = np.zeros(1, wo.SPLAT_DTYPE)[0]
    sp["x"], sp["y"], sp["dx"], sp["dy"], sp["radius"], sp["amp"] = 0.3, 0.6, 0.01, -0.02, 0.05, 400.0
    f = wo.pointer_force(n, [sp])
    assert abs(float(np.sum(f.astype(np.float64)))) < 1e-3 * float(np.sum(np.abs(f)))   # zero net circulation
    assert np.any(f != 0)


def test_spectrum_fixed_point_close_to_fp64():
    from oracle.spectral_oracle import SpectralOracle, random_field
    n = 64
    s = SpectralOracle(n=n)
    s.set_vorticity(random_field(n, k0=8, seed=2, amplitude=6.0))
    spec, e, z = wo.spectrum_fixed_point(s.w.astype(np.complex64), n)
    assert abs(e - s.energy()) < 1e-6 * n * n + 0.05 * s.energy()
    assert abs(z - s.enstrophy()) < 1e-6 * n * n + 0.05 * s.enstrophy()
