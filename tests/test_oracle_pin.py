"""Pin the CPU oracle against the reference's own golden vectors (CPU only).

* tests/golden/fixtures.npz: the reference's tests/fixtures.json (N=32),
  generated by reference/make_fixtures.py:19-80;
* tests/golden/fft_golden.npz: reference/fft_ref.py tables and line transforms;
* tests/golden/spectral_golden.npz: reference/spectral2d.py trajectories.
"""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import fft_oracle as fo
from oracle.spectral_oracle import SpectralOracle, random_field


def _oracle_from_fixture(fx):
    n = int(fx["n"])
    return SpectralOracle(n=n, beta=float(fx["beta"]), mu=float(fx["mu"]), tau=float(fx["tau"]),
                          hyper_p=int(fx["hyperP"]))


def test_fixture_fft(fixtures):
    a = fixtures["fft_input"]
    assert rel_l2(np.fft.fft2(a), fixtures["fft_forward"]) < 1e-14
    assert rel_l2(np.fft.ifft2(a), fixtures["fft_inverse"]) < 1e-14


def test_fixture_nu_h(fixtures):
    s = _oracle_from_fixture(fixtures)
    assert abs(s.nu_h / float(fixtures["nuH"]) - 1) < 1e-14


def test_fixture_velocity_packs(fixtures):
    s = _oracle_from_fixture(fixtures)
    pa, pb = s.packs(fixtures["vel_what"])
    assert rel_l2(pa, fixtures["vel_packA"]) < 1e-14
    assert rel_l2(pb, fixtures["vel_packB"]) < 1e-14


def test_fixture_assemble(fixtures):
    s = _oracle_from_fixture(fixtures)
    w = fixtures["vel_what"]
    assert rel_l2(s.product_spectrum(w), fixtures["asm_z"]) < 1e-13
    assert rel_l2(-s.unpack_nonlinear(fixtures["asm_z"]), fixtures["asm_rhs"]) < 1e-13


def test_fixture_step_and_run20(fixtures):
    s = _oracle_from_fixture(fixtures)
    s.w = fixtures["step_before"].copy()
    s.step(dt=float(fixtures["dt"]))
    assert rel_l2(s.w, fixtures["step_after"]) < 1e-13
    s.w = fixtures["step_before"].copy()
    for _ in range(20):
        s.step(dt=float(fixtures["dt"]))
    assert rel_l2(s.w, fixtures["run20_after"]) < 1e-12
    assert abs(s.energy() / float(fixtures["run20_energy"]) - 1) < 1e-12
    assert abs(s.enstrophy() / float(fixtures["run20_enstrophy"]) - 1) < 1e-12


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
def test_digit_reverse_tables(fft_golden, n):
    assert fo.radix_schedule(n) == list(fft_golden[f"radices_{n}"])
    assert np.array_equal(fo.digit_reverse_table(n), fft_golden[f"rev_{n}"])
    assert fo.is_bijective(n)


def test_radix_schedule_rejects():
    for n in (3, 6, 12, 24, 96):
        with pytest.raises(ValueError):
            fo.radix_schedule(n)


@pytest.mark.parametrize("n", [32, 64, 128, 256, 512, 1024])
def test_dit_line_model(fft_golden, n):
    x = fft_golden[f"line_in_{n}"]
    assert rel_l2(fo.dit_line(x, False), fft_golden[f"line_fwd_{n}"]) < 1e-14
    assert rel_l2(fo.dit_line(x, True), fft_golden[f"line_inv_{n}"]) < 1e-14
    assert rel_l2(fo.dit_line(x, False), np.fft.fft(x)) < 1e-13


def test_fft2_model(fft_golden):
    x = fft_golden["fft2_in_32"]
    assert rel_l2(fo.fft2_model(x), fft_golden["fft2_fwd_32"]) < 1e-14


def test_random_field_and_set_vorticity(spectral_golden):
    f = random_field(64, k0=8, seed=1)
    assert np.max(np.abs(f - spectral_golden["rf_field"])) < 1e-13
    beta, mu, tau, p, nu_h = spectral_golden["params"]
    s = SpectralOracle(n=64, beta=beta, mu=mu, tau=tau, hyper_p=int(p))
    assert abs(s.nu_h / nu_h - 1) < 1e-14
    s.set_vorticity(f)
    assert rel_l2(s.w, spectral_golden["w0"]) < 1e-14
    assert rel_l2(s.nonlinear(s.w), spectral_golden["nl0"]) < 1e-13
    assert abs(s.timestep() / float(spectral_golden["dt_cfl0"]) - 1) < 1e-13


def test_trajectory_and_diagnostics(spectral_golden):
    beta, mu, tau, p, _ = spectral_golden["params"]
    s = SpectralOracle(n=64, beta=beta, mu=mu, tau=tau, hyper_p=int(p))
    s.w = spectral_golden["w0"].copy()
    s.step(dt=0.01)
    assert rel_l2(s.w, spectral_golden["w1"]) < 1e-13
    for _ in range(9):
        s.step(dt=0.01)
    assert rel_l2(s.w, spectral_golden["w10"]) < 1e-12
    assert abs(s.energy() / float(spectral_golden["energy10"]) - 1) < 1e-12
    assert abs(s.enstrophy() / float(spectral_golden["enstrophy10"]) - 1) < 1e-12
    assert np.allclose(s.spectrum()[1], spectral_golden["spectrum10"], rtol=1e-11, atol=1e-20)
    assert np.allclose(s.zonal_mean_u(), spectral_golden["zonal10"], rtol=1e-10, atol=1e-14)


def test_laplacian_viscosity_trajectory(spectral_golden):
    s = SpectralOracle(n=64, beta=3.0, mu=0.0, tau=40.0, hyper_p=1)
    assert abs(s.nu_h / float(spectral_golden["p1_nu_h"]) - 1) < 1e-14
    s.w = spectral_golden["p1_w0"].copy()
    for _ in range(5):
        s.step(dt=0.02)
    assert rel_l2(s.w, spectral_golden["p1_w5"]) < 1e-12


def test_taylor_green(spectral_golden):
    s = SpectralOracle(n=64, beta=0.0, mu=0.0, tau=40.0, hyper_p=1)
    s.w = spectral_golden["tg_w0"].copy()
    nl = np.max(np.abs(s.nonlinear(s.w))) / np.max(np.abs(s.w))
    assert nl < 1e-14 and float(spectral_golden["tg_nl_rel"]) < 1e-14
    for _ in range(300):
        s.step(dt=0.01)
    assert rel_l2(s.w, spectral_golden["tg_w300"]) < 1e-11
    decay = abs(s.w[2, 2] / spectral_golden["tg_w0"][2, 2])
    expected = np.exp(-s.nu_h * 8.0 * 3.0)
    assert abs(decay / expected - 1) < 1e-9          # spectral2d.py:200-202
