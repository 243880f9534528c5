"""The allocation-free CFL entry point, s2d_cfl_dt_static, through the C ABI.

Callers that cannot allocate device memory (an application whose allocator owns
all GPU memory, or a frame loop that may not call cudaMalloc/cudaFree because
they can synchronize the device) pass their own device buffers and get the same
[dt, max |u|+|v|] that the solver's encodeReduce computes; the entry point's
scratch is a static device array shared by all calls.  This file is collected
last so that a stop-at-first-failure run has already run every other test.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from gpu_helpers import config
from oracle.spectral_oracle import random_field

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


@pytest.mark.parametrize("n", [32, 1024, 4096])
def test_static_scratch_cfl_matches_encode_reduce(pkg, n):
    """n = 32: one partial covers the whole field; n = 4096: every slot of the array is used."""
    torch = pytest.importorskip("torch")
    cfg = config(cfl=0.5, dtMin=1e-5, dtMax=0.02)
    rng = np.random.default_rng(5)
    for call in range(2):            # two calls in a row: the shared scratch must not leak between them
        amp = 3.0 if call == 0 else 0.5
        u = random_field(n, k0=min(16, n // 4), seed=10 + call, amplitude=amp).astype(np.float32)
        v = (amp * rng.standard_normal((n, n))).astype(np.float32)
        vel = (u + 1j * v).astype(np.complex64)
        want = _solver_dt(pkg, n, vel, cfg)
        got = _static_dt(pkg, torch, vel, n, cfg)
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=0)
        assert got[1] == np.max(np.abs(u) + np.abs(v))


def test_static_scratch_rejects_sizes_beyond_its_limit(pkg):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(4, dtype=torch.float32, device="cuda")
    for stream in (None, C.c_void_p(torch.cuda.current_stream().cuda_stream)):
        rc = pkg.lib().s2d_cfl_dt_static(C.c_void_p(buf.data_ptr()), 4097, 0.5, 1e-5, 0.02,
                                         C.c_void_p(buf.data_ptr()), stream)
        assert rc == -1
        assert b"4096" in pkg.lib().s2d_last_error()


# The child process drives CUDA through the driver API only (libcuda), the way an
# application with its own context handling does: a call with the device's primary
# context current, a call with a second context of its own current, and a call with
# the primary context current again.  The scratch address differs per context, so
# each call must use the address of the context current at the time.
_CHILD = r"""
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import __graft_entry__ as ge
lib = ge.load_package().lib()
cu = C.CDLL("libcuda.so.1")
def ok(rc, what):
    if rc != 0:
        raise SystemExit(f"{what} failed: {rc}")
ok(cu.cuInit(0), "cuInit")
dev = C.c_int()
ok(cu.cuDeviceGet(C.byref(dev), 0), "cuDeviceGet")
n, cfl, dtmin, dtmax = 256, 0.5, 1e-5, 0.02
rng = np.random.default_rng(3)
def field(scale):
    return (scale * rng.standard_normal((n, n, 2))).astype(np.float32)
def expect(vel):
    s = np.float32(np.max(np.abs(vel[..., 0]) + np.abs(vel[..., 1])))
    dx = np.float32(2.0 * np.pi / n)
    dt = np.float32(dtmax) if s <= np.float32(1e-8) else min(np.float32(dtmax), (np.float32(cfl) * dx) / s)
    return np.array([max(dt, np.float32(dtmin)), s], np.float32)
def run(vel):
    d_vel, d_out = C.c_uint64(), C.c_uint64()
    ok(cu.cuMemAlloc_v2(C.byref(d_vel), C.c_size_t(vel.nbytes)), "cuMemAlloc")
    ok(cu.cuMemAlloc_v2(C.byref(d_out), C.c_size_t(8)), "cuMemAlloc")
    ok(cu.cuMemcpyHtoD_v2(d_vel, vel.ctypes.data_as(C.c_void_p), C.c_size_t(vel.nbytes)), "HtoD")
    rc = lib.s2d_cfl_dt_static(C.c_void_p(d_vel.value), n, cfl, dtmin, dtmax, C.c_void_p(d_out.value), None)
    if rc != 0:
        raise SystemExit("s2d_cfl_dt_static: " + lib.s2d_last_error().decode())
    ok(cu.cuCtxSynchronize(), "cuCtxSynchronize")
    out = np.zeros(2, np.float32)
    ok(cu.cuMemcpyDtoH_v2(out.ctypes.data_as(C.c_void_p), d_out, C.c_size_t(8)), "DtoH")
    ok(cu.cuMemFree_v2(d_vel), "cuMemFree")
    ok(cu.cuMemFree_v2(d_out), "cuMemFree")
    return out
primary = C.c_void_p()
ok(cu.cuDevicePrimaryCtxRetain(C.byref(primary), dev), "cuDevicePrimaryCtxRetain")
ok(cu.cuCtxSetCurrent(primary), "cuCtxSetCurrent")
results = []
v1 = field(2.0); results.append((run(v1), expect(v1)))
own = C.c_void_p()
ok(cu.cuCtxCreate_v2(C.byref(own), 0, dev), "cuCtxCreate")
v2 = field(0.25); results.append((run(v2), expect(v2)))
ok(cu.cuCtxSetCurrent(primary), "cuCtxSetCurrent")
v3 = field(1.0); results.append((run(v3), expect(v3)))
ok(cu.cuCtxDestroy_v2(own), "cuCtxDestroy")
ok(cu.cuDevicePrimaryCtxRelease_v2(dev), "cuDevicePrimaryCtxRelease")
for got, want in results:
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=0)
    assert got[1] == want[1], (got, want)
print("contexts ok")
"""


def test_static_scratch_follows_the_current_context(pkg):
    res = subprocess.run([sys.executable, "-c", _CHILD, ROOT], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "contexts ok" in res.stdout
