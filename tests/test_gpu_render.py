"""Headless render (render.wgsl arithmetic as a CUDA kernel) against its CPU restatement."""
import numpy as np
import pytest

from gpu_helpers import config, current_state
from oracle import render_oracle as ro
from oracle import wgsl_oracle as wo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["dye", "vorticity", "dye over vorticity", "speed"])
def test_render_matches_restatement(pkg, mode):
    n = 128
    s = pkg.Solver.create(n=n, dyeScale=2)
    try:
        s.configure(config(viscosity=1.0, cfl=0.5, dtMax=5e-3))
        s.reset({"k0": 10, "amplitude": 6, "seed": 3, "dyePattern": "bands"})
        s.step(3, dye=True, reduce=True, graph=False)
        cfg = {"mode": mode, "exposure": 1.3, "vortScale": 0.16, "dyeGain": 1.0}
        img = s.render(cfg, width=200, height=150)
        omega = np.real(np.fft.ifft2(current_state(s).astype(np.complex128))).astype(np.float32)
        vel = s.getBuffer("vel")
        vel = np.stack([vel.real, vel.imag], -1).astype(np.float32)
        dye = wo.half_bits_to_f32(s.currentDye)
        want = ro.render(dye, omega, vel, pkg._lib.RENDER_MODES.index(mode), 1.3, 0.16, 1.0, 200, 150)
    finally:
        s.destroy()
    assert img.shape == (150, 200, 4) and img.dtype == np.uint8
    diff = np.abs(img.astype(int) - want.astype(int))
    assert np.all(img[..., 3] == 255)
    assert diff.max() <= 2, diff.max()
    assert np.mean(diff > 0) <= 0.01
    assert img[..., :3].std() > 1.0          # not a blank image


def test_render_rejects_bad_arguments(pkg):
    s = pkg.Solver.create(n=64, dyeScale=1)
    try:
        with pytest.raises(pkg.S2DError):
            s.render({"mode": "dye"}, width=0, height=10)
        img = s.render({"mode": "no such mode"}, width=8, height=8)     # render.js:65: unknown -> dye
        assert img.shape == (8, 8, 4)
    finally:
        s.destroy()
