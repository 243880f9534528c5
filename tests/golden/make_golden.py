"""Generate the golden vectors under tests/golden/ from the reference itself.

Run in a container where the reference checkout is available::

    python tests/golden/make_golden.py path/to/reference

(or set S2D_REFERENCE to the checkout and pass no argument).  It

* re-exports the reference's own golden vectors ``tests/fixtures.json``
  (N=32: fft, velocity packing, assembly, one step, twenty steps) as
  ``fixtures.npz``, after checking that the recipe of
  ``reference/make_fixtures.py:19-80`` re-run through
  ``reference/spectral2d.py`` reproduces them;
* runs ``reference/fft_ref.py`` for digit-reversal tables and line transforms
  (``fft_golden.npz``);
* runs ``reference/spectral2d.py`` at N=64 for multi-step trajectories and
  diagnostics (``spectral_golden.npz``).

Nothing at test time reads the reference: the tests read only these .npz files.
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _load(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def _cplx(flat):
    a = np.asarray(flat, np.float64)
    return a[0::2] + 1j * a[1::2]


def main(ref_root=None):
    ref_root = ref_root or os.environ.get("S2D_REFERENCE")
    if not ref_root:
        raise SystemExit("usage: make_golden.py path/to/reference  (or set S2D_REFERENCE)")
    sp = _load(os.path.join(ref_root, "reference", "spectral2d.py"), "spectral2d")
    fr = _load(os.path.join(ref_root, "reference", "fft_ref.py"), "fft_ref")
    with open(os.path.join(ref_root, "tests", "fixtures.json")) as fh:
        fx = json.load(fh)

    # ---- 1. the reference's fixtures, cross-checked against its generator recipe
    n = fx["fft"]["n"]
    rng = np.random.default_rng(11)                      # make_fixtures.py:20
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    s = sp.Spectral2D(n=n, beta=7.0, mu=0.02, tau=1.5)   # make_fixtures.py:32-33
    s.set_vorticity(sp.random_field(n, k0=6, seed=3))
    uh = 1j * s.ky * s.w * s.k2_inv
    vh = -1j * s.kx * s.w * s.k2_inv
    omega, u, v = s.unpack_fields(s.w)
    z = np.fft.fft2(u * omega + 1j * (v * omega))
    rhs = -s.nonlinear(s.w)
    before = s.w.copy()
    s.step(dt=0.011)
    s2 = sp.Spectral2D(n=n, beta=7.0, mu=0.02, tau=1.5)
    s2.w = before.copy()
    for _ in range(20):
        s2.step(dt=0.011)
    regenerated = {
        "fft_input": a, "fft_forward": np.fft.fft2(a), "fft_inverse": np.fft.ifft2(a),
        "vel_what": before, "vel_packA": before + 1j * uh, "vel_packB": vh,
        "asm_z": z, "asm_rhs": rhs, "step_before": before, "step_after": s.w,
        "run20_after": s2.w,
    }
    from_json = {
        "fft_input": _cplx(fx["fft"]["input"]), "fft_forward": _cplx(fx["fft"]["forward"]),
        "fft_inverse": _cplx(fx["fft"]["inverse"]), "vel_what": _cplx(fx["velocity"]["what"]),
        "vel_packA": _cplx(fx["velocity"]["packA"]), "vel_packB": _cplx(fx["velocity"]["packB"]),
        "asm_z": _cplx(fx["assemble"]["z"]), "asm_rhs": _cplx(fx["assemble"]["rhs"]),
        "step_before": _cplx(fx["step"]["before"]), "step_after": _cplx(fx["step"]["after"]),
        "run20_after": _cplx(fx["run20"]["after"]),
    }
    for key, val in from_json.items():
        got = regenerated[key].ravel()
        err = np.max(np.abs(got - val)) / max(np.max(np.abs(val)), 1e-300)
        assert err < 1e-12, (key, err)
    out = {k: v.reshape(n, n) for k, v in from_json.items()}
    out.update(
        n=np.int64(n), beta=np.float64(fx["step"]["beta"]), mu=np.float64(fx["step"]["mu"]),
        nuH=np.float64(fx["step"]["nuH"]), hyperP=np.int64(fx["step"]["hyperP"]),
        dt=np.float64(fx["step"]["dt"]), run20_energy=np.float64(fx["run20"]["energy"]),
        run20_enstrophy=np.float64(fx["run20"]["enstrophy"]), tau=np.float64(1.5),
    )
    np.savez_compressed(os.path.join(HERE, "fixtures.npz"), **out)

    # ---- 2. FFT model: digit reversal tables and line transforms (fft_ref.py)
    fg = {}
    for nn in (2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096):
        rad = fr.radix_schedule(nn)
        fg[f"rev_{nn}"] = np.array([fr.digit_reverse(i, rad) for i in range(nn)], np.uint32)
        fg[f"radices_{nn}"] = np.array(rad, np.int64)
    lrng = np.random.default_rng(20260815)               # fft_ref.py:89
    for nn in (32, 64, 128, 256, 512, 1024):
        x = lrng.standard_normal(nn) + 1j * lrng.standard_normal(nn)
        fg[f"line_in_{nn}"] = x
        fg[f"line_fwd_{nn}"] = fr.fft_line(x, False)
        fg[f"line_inv_{nn}"] = fr.fft_line(x, True)
    x2 = lrng.standard_normal((32, 32)) + 1j * lrng.standard_normal((32, 32))
    fg["fft2_in_32"] = x2
    fg["fft2_fwd_32"] = fr.fft2_model(x2, False)
    np.savez_compressed(os.path.join(HERE, "fft_golden.npz"), **fg)

    # ---- 3. solver trajectories and diagnostics at N=64 (spectral2d.py)
    sg = {}
    nn = 64
    field = sp.random_field(nn, k0=8, seed=1)
    sg["rf_field"] = field
    s = sp.Spectral2D(n=nn, beta=8.0, mu=0.01, tau=1.0, hyper_p=4)
    s.set_vorticity(field)
    sg["w0"] = s.w.copy()
    sg["nl0"] = s.nonlinear(s.w)
    sg["dt_cfl0"] = np.float64(s.timestep())
    s.step(dt=0.01)
    sg["w1"] = s.w.copy()
    for _ in range(9):
        s.step(dt=0.01)
    sg["w10"] = s.w.copy()
    sg["energy10"] = np.float64(s.energy())
    sg["enstrophy10"] = np.float64(s.enstrophy())
    sg["spectrum10"] = s.spectrum()[1]
    sg["zonal10"] = s.zonal_mean_u()
    sg["params"] = np.array([8.0, 0.01, 1.0, 4.0, s.nu_h])
    # Navier-Stokes viscosity, Laplacian order, with beta: 5 steps
    s = sp.Spectral2D(n=nn, beta=3.0, mu=0.0, tau=40.0, hyper_p=1)
    s.set_vorticity(sp.random_field(nn, k0=6, seed=4, amplitude=2.0))
    sg["p1_w0"] = s.w.copy()
    for _ in range(5):
        s.step(dt=0.02)
    sg["p1_w5"] = s.w.copy()
    sg["p1_nu_h"] = np.float64(s.nu_h)
    # Taylor-Green, spectral2d.py:186-202
    s = sp.Spectral2D(n=nn, beta=0.0, mu=0.0, tau=40.0, hyper_p=1)
    xs = np.arange(nn) * 2 * np.pi / nn
    gx, gy = np.meshgrid(xs, xs, indexing="xy")
    s.set_vorticity(4.0 * np.cos(2 * gx) * np.cos(2 * gy))
    sg["tg_w0"] = s.w.copy()
    sg["tg_nl_rel"] = np.float64(np.max(np.abs(s.nonlinear(s.w))) / np.max(np.abs(s.w)))
    for _ in range(300):
        s.step(dt=0.01)
    sg["tg_w300"] = s.w.copy()
    sg["tg_nu_h"] = np.float64(s.nu_h)
    np.savez_compressed(os.path.join(HERE, "spectral_golden.npz"), **sg)
    for f in ("fixtures.npz", "fft_golden.npz", "spectral_golden.npz"):
        p = os.path.join(HERE, f)
        print(f"wrote {f}: {os.path.getsize(p) / 1024:.1f} KB")


if __name__ == "__main__":
    main(*sys.argv[1:])
