"""Failure detection on the device without a GPU fault.

Every device-side wait of the library (bulk-copy and MMA barriers) is bounded by a
global-timer limit; a wait that gives up records its site in the solver's error word
and lets its kernel return, and the host reports it as S2D_ERR_CUDA at the next
synchronization.  The probe entry point enqueues one CTA whose barrier expects bytes
that are never sent, so the wait runs out every time: nothing traps, nothing faults,
and the context stays usable.
"""
import time

import numpy as np
import pytest

from conftest import rel_l2
from gpu_helpers import config, current_state, load_state, set_fixed_dt
from oracle.spectral_oracle import SpectralOracle, random_field

pytestmark = pytest.mark.gpu


def _one_step_error(pkg, n=64, dt=0.01):
    ref = SpectralOracle(n=n)
    ref.set_vorticity(random_field(n, k0=8, seed=2, amplitude=2.0))
    w_in = ref.w.astype(np.complex64)
    ref.w = w_in.astype(np.complex128)
    ref.step(dt=dt)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config())
        load_state(s, w_in)
        set_fixed_dt(s, dt)
        s.setSplats([])
        s.encodeStep()
        s.synchronize()
        return rel_l2(current_state(s), ref.w)
    finally:
        s.destroy()


@pytest.mark.parametrize("limit_ns", [5_000, 2_000_000])
def test_bounded_wait_gives_up_and_is_reported(pkg, limit_ns):
    s = pkg.Solver.create(n=64, dyeScale=1)
    try:
        s.synchronize()                       # nothing pending before the probe
        t0 = time.perf_counter()
        s.probeWaitTimeout(limit_ns)
        with pytest.raises(pkg.S2DError) as info:
            s.synchronize()
        elapsed = time.perf_counter() - t0
        assert info.value.status == -3        # S2D_ERR_CUDA
        assert "site 5" in str(info.value)
        assert elapsed >= 0.9 * limit_ns * 1e-9
        assert elapsed < 5.0                  # the wait ended by itself
        s.synchronize()                       # the error word was cleared by the report
    finally:
        s.destroy()
    # the context is still usable: a fresh solver steps and matches the FP64 oracle
    assert _one_step_error(pkg) <= 1e-5


def test_probe_rejects_bad_limits(pkg):
    s = pkg.Solver.create(n=64, dyeScale=1)
    try:
        for bad in (0, 2_000_000_000):
            with pytest.raises(pkg.S2DError) as info:
                s.probeWaitTimeout(bad)
            assert info.value.status == -1
        s.synchronize()
    finally:
        s.destroy()
