"""Scenario presets (src/scenarios.js) built on the device: field against the CPU
restatement, the seeded state against the masked FFT of that field, and the device
reset equal bit for bit to reset({field}) with the same field."""
import numpy as np
import pytest

from conftest import rel_l2
from gpu_helpers import current_state
from oracle import scenarios_oracle as so
from oracle.spectral_oracle import SpectralOracle

pytestmark = pytest.mark.gpu

CASES = [("shear layer", None), ("taylor-green", None), ("dipole", None), ("merger", {"mergerSep": 0.9}),
         ("polygon", {"polygonN": 7}), ("merger", None), ("polygon", None)]


@pytest.mark.parametrize("name,cfg", CASES, ids=[f"{c[0]}-{c[1]}" for c in CASES])
def test_scenario_field_and_reset(pkg, name, cfg):
    n = 256
    want = so.build(name, n, cfg)
    s = pkg.Solver.create(n=n, dyeScale=1)
    try:
        got = s.scenarioField(name, cfg)
        scale = np.max(np.abs(want))
        assert np.max(np.abs(got - want)) <= 1e-6 * scale          # FP64 math, FP32 rounding
        s.resetScenario(name, cfg, dyePattern="bands")
        dev = current_state(s)
        assert s.phase == 0 and s.stepIndex == 0
        ref = SpectralOracle(n=n)
        ref.set_vorticity(want.astype(np.float64))       # FFT, dealias mask, k = 0 removed
        assert rel_l2(dev, ref.w) <= 1e-6
        s.reset({"field": got, "dyePattern": "bands"})
        assert np.array_equal(current_state(s), dev)
    finally:
        s.destroy()


def test_scenario_configs_mirror_the_reference(pkg):
    assert pkg.SCENARIO_NAMES == ["shear layer", "taylor-green", "dipole", "merger", "polygon"]
    assert pkg.SCENARIOS["taylor-green"]["config"]["viscosity"] == 90
    assert pkg.SCENARIOS["polygon"]["config"]["substeps"] == 8


def test_scenario_rejects_bad_parameters(pkg):
    s = pkg.Solver.create(n=64, dyeScale=1)
    try:
        with pytest.raises(pkg.S2DError) as ei:
            s.scenarioField("polygon", {"polygonN": 0})
        assert ei.value.status == -1
        with pytest.raises(pkg.S2DError):
            s.resetScenario("polygon", {"polygonN": 1000})
        with pytest.raises(ValueError):
            s.scenarioField("vortex street")
    finally:
        s.destroy()
