"""The Node-API addon (spectral-2d-turbulence_b200/napi) against the C ABI and the
reference's JavaScript Solver interface.

Node and its headers are not installed where these tests run, so the addon is not
compiled here; these checks hold its source to the library it binds: every s2d_*
function it calls is declared in include/s2d.h and exported by libs2d.so, every
native function the JS facade calls is registered by the addon, and the facade class
has every method and accessor of solver.js's Solver (src/gpu/solver.js:49-630).
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NAPI = os.path.join(ROOT, "spectral-2d-turbulence_b200", "napi")

# solver.js:71-614 -- the Solver methods and accessors callers use (main.js, tests/index.html)
REFERENCE_METHODS = ["create", "configure", "setSplats", "seed", "seedPhysical", "reset", "paintDye",
                     "encodePrime", "encodeStep", "encodeDye", "encodeReduce", "encodeDiagnostics",
                     "copyDiagnostics", "readDiagnostics", "currentDye", "destroy"]
REFERENCE_FIELDS = ["phase", "dyeParity", "stepIndex", "simTime", "primed", "paramsF"]


def _read(name):
    with open(os.path.join(NAPI, name)) as fh:
        return fh.read()


def test_addon_calls_only_declared_exported_functions(pkg):
    src = _read("s2d_napi.c")
    with open(os.path.join(ROOT, "include", "s2d.h")) as fh:
        header = fh.read()
    called = set(re.findall(r"\b(s2d_[a-z0-9_]+)\s*\(", src))
    assert called, "no C ABI calls found"
    declared = set(re.findall(r"\b(s2d_[a-z0-9_]+)\s*\(", header))
    lib = pkg.lib()
    for fn in sorted(called):
        assert fn in declared, f"{fn} is not declared in include/s2d.h"
        assert hasattr(lib, fn), f"{fn} is not exported by libs2d.so"


def test_facade_uses_registered_native_functions():
    src = _read("s2d_napi.c")
    registered = set(re.findall(r'\{"([A-Za-z0-9]+)", NULL, js_', src))
    used = set(re.findall(r"\baddon\.([A-Za-z0-9]+)\(", _read("solver_b200.js")))
    used |= set(re.findall(r"\baddon\.([A-Za-z0-9]+)\(", _read("headless.js")))
    assert used, "the facade calls no native function"
    assert used <= registered, f"unregistered native functions: {sorted(used - registered)}"


@pytest.mark.parametrize("name", REFERENCE_METHODS + REFERENCE_FIELDS)
def test_facade_has_reference_member(name):
    js = _read("solver_b200.js")
    pattern = rf"^\s*(static\s+async\s+|async\s+|get\s+|set\s+)?{name}\s*\("
    assert re.search(pattern, js, re.M), f"Solver.{name} missing from solver_b200.js"


def test_binding_builds_the_addon_against_the_library():
    gyp = _read("binding.gyp")
    assert '"s2d_napi.c"' in gyp and "-ls2d" in gyp and "../../include" in gyp
    assert "solver_b200.js" in _read("package.json")
