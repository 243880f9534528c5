"""Stage-kernel shapes and the autotuner: every registered shape matches the FP64 oracle,
autotuning leaves the solver's state untouched and later solvers reuse its choice."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_helpers import config, current_state, load_state, rate_for, set_fixed_dt
from oracle.spectral_oracle import SpectralOracle, random_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [512, 1024])
def test_every_registered_shape_matches_oracle(pkg, n):
    beta, mu, p, dt = 10.0, 1e-2, 4, 1e-3
    nu_h = 1.0 / (n / 3.0) ** 8
    ref0 = SpectralOracle(n=n, beta=beta, mu=mu, nu_h=nu_h, hyper_p=p)
    ref0.set_vorticity(random_field(n, k0=n / 8, seed=n + 3, amplitude=8.0))
    w_in = ref0.w.astype(np.complex64)
    ref0.w = w_in.astype(np.complex128)
    ref0.step(dt=dt)
    want = ref0.w
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        rep = s.autotune(steps=3)
        ncol, nrow = len(rep["column"]), len(rep["row"])
        assert ncol >= 2 and nrow >= 2            # the V=8 shapes are registered at these sizes
        s.configure(config(beta=beta, drag=mu, viscosity=rate_for(nu_h, n, p), hyperP=p))
        for i in range(ncol):
            for j in range(nrow):
                s.tuneSelect(i, j)
                load_state(s, w_in)
                set_fixed_dt(s, dt)
                s.encodeStep()
                err = rel_l2(current_state(s), want)
                assert err <= 1e-5, (rep["column"][i][0], rep["row"][j][0], err)
    finally:
        s.destroy()


def test_autotune_restores_state_and_is_remembered(pkg):
    n = 1024
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        s.configure(config(viscosity=1.0, hyperP=4, forceAmp=0.1, forceK=64.0, forceWidth=2.0, cfl=0.5,
                           dtMax=1e-3))
        s.reset({"k0": 14, "amplitude": 6, "seed": 1, "dyePattern": "none"})
        s.step(2, dye=False, reduce=True)
        before = (current_state(s), s.getBuffer("dt"), s.getBuffer("vel"), s.phase, s.stepIndex)
        rep = s.autotune(steps=5)
        after = (current_state(s), s.getBuffer("dt"), s.getBuffer("vel"), s.phase, s.stepIndex)
        assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
        assert np.array_equal(before[2], after[2]) and before[3:] == after[3:]
        assert all(us > 0 for _, us in rep["column"]) and all(us > 0 for _, us in rep["row"])
        best_row = min(rep["row"], key=lambda kv: kv[1])[0]
        assert rep["choice"]["row"] == best_row
        # stepping on with the chosen shapes
        s.step(2, dye=False, reduce=True, graph=True)
        assert np.all(np.isfinite(current_state(s)))
    finally:
        s.destroy()
    s2 = pkg.Solver.create(n=n, dyeScale=1)
    try:
        again = s2.autotune(steps=1)          # a new solver starts from the remembered choice
        assert again["choice"]["row"] in [name for name, _ in again["row"]]
    finally:
        s2.destroy()


def _mixed_ensemble(pkg):
    inst = []
    for n, count in ((64, 3), (128, 2), (256, 2)):
        for k in range(count):
            inst.append({"n": n, "beta": 5.0 + k, "drag": 1e-2, "nuH": 5e-4, "hyperP": 1, "dt": 2e-3,
                         "seed": len(inst)})
    e = pkg.Ensemble(inst)
    e.seedBand(4.0, 12.0, rms=1.0)
    return e


def test_ensemble_autotune_restores_state_and_matches(pkg):
    e = _mixed_ensemble(pkg)
    ref = _mixed_ensemble(pkg)
    try:
        e.step(2, graph=False)
        ref.step(2, graph=False)
        before = [e.getState(i) for i in range(e.count)]
        rep = e.autotune(2)
        assert len(rep["column"]) == 2 and len(rep["row"]) == 4
        assert all(us > 0 for _, us in rep["column"] + rep["row"])
        for i in range(e.count):
            assert np.array_equal(e.getState(i), before[i])
        e.step(6, graph=True)
        ref.step(6, graph=True)
        for i in range(e.count):
            a, b = e.getState(i), ref.getState(i)
            assert rel_l2(a, b) <= 1e-6, i
    finally:
        e.destroy()
        ref.destroy()


@pytest.mark.parametrize("n,suffix", [(512, "staged rows"), (1024, "paired inverse transforms")])
def test_derived_row_shape_matches_its_twin(pkg, n, suffix):
    """A row shape derived from another one, with pointer forcing and stochastic forcing
    on.  Staging wcur / w0 / pointer force by bulk copy changes only where the same values
    are loaded from: the states agree bit for bit.  Running the two inverse transforms
    of the next packs as one two-line transform is the same arithmetic, but the compiler
    may contract its multiply-adds differently: the states agree to FP32 rounding."""
    splat = {"x": 0.3, "y": 0.6, "dx": 0.02, "dy": -0.01, "color": (1.0, 0.5, 0.2), "radius": 0.04,
             "amp": 3.0, "dyeAmp": 0.5}
    outs = []
    for staged in (False, True):
        s = pkg.Solver.create(n=n, dyeScale=1)
        try:
            rep = s.autotune(steps=1)
            names = [name for name, _ in rep["row"]]
            twin = next(i for i, nm in enumerate(names) if nm.endswith(suffix))
            plain = names.index(names[twin].replace(", " + suffix, ""))
            s.tuneSelect(0, twin if staged else plain)
            s.configure(config(beta=5.0, drag=1e-2, viscosity=1.0, hyperP=4, forceAmp=0.2, forceK=n / 16,
                               forceWidth=2.0, cfl=0.5, dtMax=1e-3))
            s.reset({"k0": 10, "amplitude": 6, "seed": 5, "dyePattern": "none"})
            s.setSplats([splat])
            s.step(3, dye=False, reduce=True, graph=False, relatch=True)
            s.setSplats([])
            s.step(2, dye=False, reduce=True, graph=True, relatch=True)
            outs.append((current_state(s), s.getBuffer("packA"), s.getBuffer("dt")))
        finally:
            s.destroy()
    if suffix == "staged rows":
        for a, b in zip(outs[0], outs[1]):
            assert np.array_equal(a, b)
    else:
        assert rel_l2(outs[1][0], outs[0][0]) <= 1e-6
        assert rel_l2(outs[1][1], outs[0][1]) <= 1e-6
        assert abs(float(outs[1][2][0]) / float(outs[0][2][0]) - 1.0) <= 1e-5


def test_every_ensemble_shape_matches_the_default(pkg):
    """Each registered launch shape of the persistent ensemble kernels (resident CTAs,
    paired inverse transforms) steps the mixed ensemble like the default shape, to FP32
    rounding (the paired transform may contract multiply-adds differently)."""
    ref = _mixed_ensemble(pkg)
    try:
        ref.step(4, graph=True)
        want = [ref.getState(i) for i in range(ref.count)]
        rep = ref.autotune(1)
        names = [nm for nm, _ in rep["row"]]
        assert any(nm.endswith("paired inverse transforms") for nm in names)
    finally:
        ref.destroy()
    for col in range(len(rep["column"])):
        for row in range(len(rep["row"])):
            e = _mixed_ensemble(pkg)
            try:
                e.tuneSelect(col, row)
                e.step(4, graph=True)
                for i in range(e.count):
                    assert rel_l2(e.getState(i), want[i]) <= 1e-6, (rep["column"][col][0], names[row], i)
            finally:
                e.destroy()
