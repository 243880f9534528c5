"""The reference's browser harness (tests/index.html:114-203), through the C ABI.

Same inputs (tests/fixtures.json of the reference, N=32), same checks, same
L-infinity relative metric and tolerances, plus tighter relative-L2 bounds.
"""
import numpy as np
import pytest

from conftest import rel_l2, rel_linf
from gpu_helpers import config

pytestmark = pytest.mark.gpu


@pytest.fixture
def solver(pkg, fixtures):
    n = int(fixtures["n"])
    s = pkg.Solver.create(n=n, dyeScale=1)
    s.configure(config(beta=float(fixtures["beta"]), drag=float(fixtures["mu"]), viscosity=1 / 1.5,
                       hyperP=int(fixtures["hyperP"]), forceAmp=0.0, forceK=20.0, forceWidth=2.0,
                       cfl=0.5, dtMin=1e-6, dtMax=1.0, dyeFade=1.0))
    yield s
    s.destroy()


def test_nu_h_coefficient(solver, fixtures):
    assert abs(solver.paramsF[2] / float(fixtures["nuH"]) - 1) <= 1e-6          # index.html:136-140


def test_fft2_forward_inverse(solver, fixtures):
    solver.setBuffer("packA", fixtures["fft_input"])
    solver.fft.forward(None, "packA")
    got = solver.getBuffer("packA")
    assert rel_linf(got, fixtures["fft_forward"]) <= 2e-5                       # index.html:151
    assert rel_l2(got, fixtures["fft_forward"]) <= 1e-6
    solver.setBuffer("packA", fixtures["fft_input"])
    solver.fft.inverse(None, "packA")
    got = solver.getBuffer("packA")
    assert rel_linf(got, fixtures["fft_inverse"]) <= 2e-5                       # index.html:159
    assert rel_l2(got, fixtures["fft_inverse"]) <= 1e-6


def test_velocity_packing(solver, fixtures):
    solver.setBuffer("state0", fixtures["vel_what"])
    solver.phase = 0
    solver.velocityPack(0)
    assert rel_linf(solver.getBuffer("packA"), fixtures["vel_packA"]) <= 2e-5   # index.html:170
    assert rel_linf(solver.getBuffer("packB"), fixtures["vel_packB"]) <= 2e-5   # index.html:171


def test_nonlinear_assembly(solver, fixtures):
    solver.setBuffer("physZ", fixtures["asm_z"])
    solver.setBuffer("force", np.zeros_like(fixtures["asm_z"]))
    solver.assemble()
    got = solver.getBuffer("rhs")
    assert rel_linf(got, fixtures["asm_rhs"]) <= 5e-5                           # index.html:182
    assert rel_l2(got, fixtures["asm_rhs"]) <= 1e-6


def _run_steps(solver, fixtures, count, fused=True):
    solver.phase = 0
    solver.dyeParity = 0
    solver.setBuffer("state0", fixtures["step_before"])
    solver.setBuffer("dt", np.array([float(fixtures["dt"]), 0, 0, 0], np.float32))
    solver.setSplats([])
    for _ in range(count):
        if fused:
            solver.encodeStep()
        else:
            solver.encodeStepUnfused()
    return solver.getBuffer(f"state{solver.phase}")


@pytest.mark.parametrize("fused", [True, False], ids=["fused", "reference-order"])
def test_one_rk3_step(solver, fixtures, fused):
    got = _run_steps(solver, fixtures, 1, fused)
    assert rel_linf(got, fixtures["step_after"]) <= 5e-5                        # index.html:200
    assert rel_l2(got, fixtures["step_after"]) <= 1e-5


@pytest.mark.parametrize("fused", [True, False], ids=["fused", "reference-order"])
def test_twenty_steps(solver, fixtures, fused):
    got = _run_steps(solver, fixtures, 20, fused)
    assert rel_linf(got, fixtures["run20_after"]) <= 5e-3                       # index.html:201
    assert rel_l2(got, fixtures["run20_after"]) <= 1e-4
    solver.encodeDiagnostics()
    solver.copyDiagnostics()
    d = solver.readDiagnostics()
    assert abs(d["energy"] / float(fixtures["run20_energy"]) - 1) <= 1e-4
    assert abs(d["enstrophy"] / float(fixtures["run20_enstrophy"]) - 1) <= 1e-4
