"""Batched uneven ensemble vs per-instance oracle runs; error behaviour."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_helpers import config
from oracle.spectral_oracle import SpectralOracle

pytestmark = pytest.mark.gpu


def _instances():
    rng = np.random.default_rng(42)
    out = []
    for n, count in ((64, 3), (128, 2), (256, 2), (512, 1), (1024, 1)):   # every accepted size, 64..1024
        for _ in range(count):
            out.append({"n": n, "beta": float(rng.uniform(0, 20)), "drag": float(rng.uniform(0, 2e-2)),
                        "nuH": float(rng.uniform(1e-4, 1e-3)), "hyperP": 1, "dt": 2e-3,
                        "seed": int(rng.integers(1 << 30))})
    out.append({"n": 128, "beta": 3.0, "drag": 0.01, "nuH": 1e-14, "hyperP": 4, "dt": 1e-3,
                "forceAmp": 0.1, "forceK": 20.0, "forceWidth": 2.0, "seed": 5})
    return out


def test_ensemble_matches_oracle_per_instance(pkg):
    inst = _instances()
    e = pkg.Ensemble(inst)
    try:
        e.seedBand(4.0, 12.0, rms=1.0)
        w0 = [e.getState(i) for i in range(e.count)]
        for i, w in enumerate(w0):
            n = inst[i]["n"]
            assert abs(np.sqrt(np.sum(np.abs(w.astype(np.complex128)) ** 2)) / (n * n) - 1) < 1e-5
        steps = 4
        e.step(steps, graph=True)
        for i, d in enumerate(inst):
            if d.get("forceAmp", 0) > 0:
                continue
            ref = SpectralOracle(n=d["n"], beta=d["beta"], mu=d["drag"], nu_h=d["nuH"], hyper_p=d["hyperP"])
            ref.w = w0[i].astype(np.complex128)
            for _ in range(steps):
                ref.step(dt=d["dt"])
            err = rel_l2(e.getState(i), ref.w)
            assert err <= 2e-5, (i, d["n"], err)
        en, ens = e.energy()
        for i, d in enumerate(inst):
            ref = SpectralOracle(n=d["n"])
            ref.w = e.getState(i).astype(np.complex128)
            assert abs(en[i] / ref.energy() - 1) < 1e-12
            assert abs(ens[i] / ref.enstrophy() - 1) < 1e-12
    finally:
        e.destroy()


def test_ensemble_graph_equals_direct_launches(pkg):
    inst = _instances()
    results = []
    for graph in (True, False):
        e = pkg.Ensemble(inst)
        try:
            e.seedBand(4.0, 12.0, rms=1.0)
            e.step(7, graph=graph)
            results.append([e.getState(i) for i in range(e.count)])
        finally:
            e.destroy()
    for a, b in zip(*results):
        assert np.array_equal(a, b)


def test_ensemble_matches_single_solver(pkg):
    inst = [{"n": 256, "beta": 5.0, "drag": 0.01, "nuH": 1e-14, "hyperP": 4, "dt": 1e-3, "seed": 11,
             "forceAmp": 0.1, "forceK": 30.0, "forceWidth": 2.0}]
    e = pkg.Ensemble(inst)
    s = pkg.Solver.create(n=256, dyeScale=1)
    try:
        e.seedBand(4.0, 12.0)
        w0 = e.getState(0)
        s.configure(config(beta=5.0, drag=0.01, viscosity=1e-14 * (256 / 3.0) ** 8, hyperP=4, forceAmp=0.1,
                           forceK=30.0, forceWidth=2.0))
        s.phase = 0
        s.setBuffer("state0", w0)
        s.setBuffer("dt", np.array([1e-3, 0, 0, 0], np.float32))
        e.step(1, graph=False)
        s.encodeStep()
        assert rel_l2(e.getState(0), s.getBuffer(f"state{s.phase}")) <= 1e-6
    finally:
        e.destroy()
        s.destroy()


def test_ensemble_rejects_bad_sizes(pkg):
    with pytest.raises(pkg.S2DError) as ei:
        pkg.Ensemble([{"n": 96, "dt": 1e-3}])
    assert ei.value.status == -2
    with pytest.raises(pkg.S2DError):
        pkg.Ensemble([{"n": 2048, "dt": 1e-3}])


# ---------------------------------------------------------------- errors
@pytest.mark.parametrize("n", [48, 16, 8192, 0])
def test_unsupported_grid(pkg, n):
    with pytest.raises(pkg.S2DError) as ei:
        pkg.Solver.create(n=n)
    assert ei.value.status == -2


def test_use_after_destroy(pkg):
    s = pkg.Solver.create(n=64, dyeScale=1)
    s.destroy()
    with pytest.raises(pkg.S2DError) as ei:
        s.encodeStep()
    assert ei.value.status == -4
    assert s.readDiagnostics() is None                                      # solver.js:571


def test_nan_field_rejected(pkg):
    s = pkg.Solver.create(n=64, dyeScale=1)
    try:
        f = np.zeros((64, 64), np.float32)
        f[3, 5] = np.nan
        with pytest.raises(pkg.S2DError) as ei:
            s.seedPhysical(f)
        assert ei.value.status == -5
        w = np.zeros((64, 64), np.complex64)
        w[1, 1] = np.inf
        with pytest.raises(pkg.S2DError) as ei:
            s.setBuffer("state0", w)
        assert ei.value.status == -5
    finally:
        s.destroy()


def test_supported_grids(pkg):
    grids = pkg.supportedGrids()
    assert grids == [32, 64, 128, 256, 512, 1024, 2048, 4096]
