"""The allocation-free CFL entry point, s2d_cfl_dt_static, through the C ABI.

Callers that cannot allocate device memory (an application whose allocator owns
all GPU memory, or a frame loop that may not call cudaMalloc/cudaFree because
they can synchronize the device) pass their own device buffers and get the same
[dt, max |u|+|v|] that the solver's encodeReduce computes; the entry point's
scratch is a static device array shared by all calls.  This file is collected
last so that a stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_helpers import config
from oracle.spectral_oracle import random_field

pytestmark = pytest.mark.gpu


def _solver_dt(pkg, n, vel, cfg):
    """[dt, speed] from the existing entry point (Solver.encodeReduce) for velocity `vel`."""
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(cfg)
        s.setBuffer("vel", vel)
        s.encodeReduce()
        return s.getBuffer("dt")[:2]
    finally:
        s.destroy()


def _static_dt(pkg, torch, vel, n, cfg):
    dev_vel = torch.from_numpy(np.ascontiguousarray(vel).view(np.float32).reshape(-1)).cuda()
    out = torch.full((2,), -1.0, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = pkg.lib().s2d_cfl_dt_static(C.c_void_p(dev_vel.data_ptr()), n, cfg["cfl"], cfg["dtMin"], cfg["dtMax"],
                                     C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert rc == 0, pkg.lib().s2d_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_static_scratch_cfl_matches_encode_reduce(pkg):
    torch = pytest.importorskip("torch")
    n = 1024
    cfg = config(cfl=0.5, dtMin=1e-5, dtMax=0.02)
    rng = np.random.default_rng(5)
    for call in range(2):            # two calls in a row: the shared scratch must not leak between them
        amp = 3.0 if call == 0 else 0.5
        u = random_field(n, k0=16, seed=10 + call, amplitude=amp).astype(np.float32)
        v = (amp * rng.standard_normal((n, n))).astype(np.float32)
        vel = (u + 1j * v).astype(np.complex64)
        want = _solver_dt(pkg, n, vel, cfg)
        got = _static_dt(pkg, torch, vel, n, cfg)
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=0)
        assert got[1] == np.max(np.abs(u) + np.abs(v))


def test_static_scratch_rejects_sizes_beyond_its_limit(pkg):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(4, dtype=torch.float32, device="cuda")
    rc = pkg.lib().s2d_cfl_dt_static(C.c_void_p(buf.data_ptr()), 4097, 0.5, 1e-5, 0.02,
                                     C.c_void_p(buf.data_ptr()), None)
    assert rc == -1
    assert b"4096" in pkg.lib().s2d_last_error()
