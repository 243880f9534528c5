"""Host-side ``Solver``: the reference's JavaScript solver API over the C ABI.

Method names, argument meaning and error behaviour follow
``src/gpu/solver.js`` (class Solver, lines 49-630) and ``src/gpu/fft.js``
(radixSchedule, Fft2D), so code written against the reference reads the same:

    solver = Solver.create(n=256, dyeScale=2)
    solver.configure(cfg)                 # cfg keys as main.js:9-36
    solver.reset({"k0": 14, "amplitude": 6, "seed": 1})
    solver.encodePrime()
    for _ in range(substeps):
        solver.encodeStep(); solver.encodeDye(); solver.encodeReduce()
    solver.encodeDiagnostics(); solver.copyDiagnostics()
    diag = solver.readDiagnostics()       # dict or None, like the JS promise

Every GPU operation is enqueued on the solver's CUDA stream in call order (the
``pass`` / ``encoder`` arguments of the JS methods are accepted and ignored).
Negative C statuses raise ``S2DError`` where the JS throws.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

MAX_SPLATS = L.S2D_MAX_SPLATS   # solver.js:9
_PRECISIONS = {"fp32": L.S2D_FFT_FP32, "tc-f16": L.S2D_FFT_TC_F16, "tc-bf16": L.S2D_FFT_TC_BF16}
_PATTERNS = {"none": L.S2D_DYE_NONE, "bands": L.S2D_DYE_BANDS}


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def radixSchedule(n: int) -> dict:
    """fft.js:20-31: {'stages', 'hasRadix2'}; raises for n not 4^a or 2*4^a."""
    st, r2 = C.c_int(), C.c_int()
    L.call("s2d_radix_schedule", int(n), C.byref(st), C.byref(r2))
    return {"stages": st.value, "hasRadix2": bool(r2.value)}


def supportedGrids() -> list[int]:
    """device.js:44-52, re-derived from this GPU's shared memory and HBM."""
    out = (C.c_int * 16)()
    cnt = C.c_int()
    L.call("s2d_supported_grids", out, 16, C.byref(cnt))
    return [out[i] for i in range(min(cnt.value, 16))]


def digitReverseTable(n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    L.call("s2d_digit_reverse_table", int(n), out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out


def wavenumberTable(n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    L.call("s2d_wavenumber_table", int(n), _fptr(out))
    return out


def dealiasMaskTable(n: int) -> np.ndarray:
    out = np.zeros((n, n), np.uint8)
    L.call("s2d_dealias_mask_table", int(n), out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return out


class Fft2D:
    """fft.js:33-101 over the solver's registered buffers (packA, packB, physZ, force)."""

    def __init__(self, solver: "Solver"):
        self._s = solver
        self.n = solver.n

    def run(self, pass_, name: str, inverse: bool):
        bid = L.BUFFER_IDS.get(name, -1)
        if bid < 0:
            raise L.S2DError(L.S2D_ERR_UNREGISTERED, "Fft2D.run",
                             f"buffer {name} was never registered with the FFT")
        L.call("s2d_fft2", self._s._h, bid, 1 if inverse else 0)

    def forward(self, pass_, name: str):
        self.run(pass_, name, False)

    def inverse(self, pass_, name: str):
        self.run(pass_, name, True)


class Solver:
    """GPU pseudo-spectral vorticity solver (solver.js:49-630)."""

    def __init__(self, handle, n, dye_scale, device):
        self._h = handle
        self.n = n
        self.ncells = n * n
        self.m = n * dye_scale
        self.nbins = n // 2 + 1
        self.device = device
        self.cfg = None
        self.disposed = False
        self.fft = Fft2D(self)

    # ---------------------------------------------------------------- lifecycle
    @staticmethod
    def create(device: int = 0, n: int = 256, dyeScale: int = 2, fft: str = "fp32") -> "Solver":
        """solver.js:71-75 (``create(device, {n, dyeScale})``); ``fft`` selects the FFT arithmetic:
        "fp32" (CUDA cores, every size) or the tensor-core split forms "tc-f16" / "tc-bf16"
        (N = 256, 512, 1024, 2048, 4096; fused stage kernels at 1024^2, the reference's
        per-stage order with tensor-core 2D transforms at the other sizes)."""
        if fft not in _PRECISIONS:
            raise ValueError(f"unknown FFT arithmetic {fft!r}")
        h = C.c_void_p()
        L.call("s2d_create", int(n), int(dyeScale), _PRECISIONS[fft], int(device), C.byref(h))
        return Solver(h, int(n), int(dyeScale), int(device))

    def destroy(self):
        """solver.js:614-629; later calls raise (use after destroy)."""
        if not self.disposed:
            L.call("s2d_destroy", self._h)
            self.disposed = True
            self._h = None

    def _use(self):
        if self.disposed:
            raise L.S2DError(L.S2D_ERR_DESTROYED, "Solver", "solver destroyed")
        return self._h

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # ---------------------------------------------------------------- state fields
    def _info(self) -> L.s2d_info:
        i = L.s2d_info()
        L.call("s2d_get_info", self._use(), C.byref(i))
        return i

    @property
    def phase(self) -> int:
        return self._info().phase

    @phase.setter
    def phase(self, v: int):
        L.call("s2d_set_phase", self._use(), int(v), self._info().dye_parity)

    @property
    def dyeParity(self) -> int:
        return self._info().dye_parity

    @dyeParity.setter
    def dyeParity(self, v: int):
        L.call("s2d_set_phase", self._use(), self._info().phase, int(v))

    @property
    def stepIndex(self) -> int:
        return self._info().step_index

    @property
    def primed(self) -> bool:
        return bool(self._info().primed)

    @property
    def simTime(self) -> float:
        return self._info().sim_time

    @simTime.setter
    def simTime(self, t: float):
        L.call("s2d_set_sim_time", self._use(), float(t))

    @property
    def paramsF(self) -> np.ndarray:
        """The 12-float Params view (solver.js:63-65); index 2 is nuH."""
        i = self._info()
        c = self.cfg or {}
        out = np.zeros(12, np.float32)
        out[0] = c.get("beta", 0.0)
        out[1] = c.get("drag", 0.0)
        out[2] = i.nu_h
        out[3] = c.get("hyperP", 0)
        out[4] = c.get("forceAmp", 0.0)
        out[5] = c.get("forceK", 0.0)
        out[6] = c.get("forceWidth", 0.0)
        out[7] = np.uint32(i.step_index).view(np.float32)
        out[8] = 2 * np.pi / self.n
        out[9] = c.get("cfl", 0.0)
        out[10] = c.get("dtMin", 0.0)
        out[11] = c.get("dtMax", 0.0)
        return out

    @property
    def stream(self) -> int:
        """The cudaStream_t every call of this solver is ordered on (as an int)."""
        p = C.c_void_p()
        L.call("s2d_get_stream", self._use(), C.byref(p))
        return p.value or 0

    def synchronize(self):
        L.call("s2d_synchronize", self._use())

    def probeWaitTimeout(self, limit_ns: int):
        """Enqueue one CTA whose bounded device wait cannot complete (failure-detection
        check): the next synchronize() raises S2DError with S2D_ERR_CUDA."""
        L.call("s2d_probe_wait_timeout", self._use(), int(limit_ns))

    # ---------------------------------------------------------------- parameters
    def configure(self, cfg: dict):
        """solver.js:306-324: latches stepIndex for the stochastic forcing phase."""
        p = L.s2d_params(
            beta=float(cfg["beta"]), drag=float(cfg["drag"]), viscosity=float(cfg["viscosity"]),
            hyper_p=int(cfg["hyperP"]), force_amp=float(cfg["forceAmp"]), force_k=float(cfg["forceK"]),
            force_width=float(cfg["forceWidth"]), cfl=float(cfg["cfl"]), dt_min=float(cfg["dtMin"]),
            dt_max=float(cfg["dtMax"]), dye_fade=float(cfg["dyeFade"]))
        L.call("s2d_configure", self._use(), C.byref(p))
        self.cfg = dict(cfg)

    def setSplats(self, splats):
        """solver.js:326-345: at most MAX_SPLATS entries are used."""
        splats = list(splats)[:MAX_SPLATS]
        arr = (L.s2d_splat * max(1, len(splats)))()
        for i, s in enumerate(splats):
            arr[i].x, arr[i].y = s["x"], s["y"]
            arr[i].dx, arr[i].dy = s["dx"], s["dy"]
            for c in range(3):
                arr[i].color[c] = s["color"][c]
            arr[i].radius, arr[i].amp, arr[i].dye_amp = s["radius"], s["amp"], s["dyeAmp"]
        L.call("s2d_set_splats", self._use(), arr, len(splats))

    # ---------------------------------------------------------------- seeding
    def seed(self, k0: float = 14, amplitude: float = 6, seed: int = 1):
        """solver.js:347-359 (fillSpectrum, 384-418)."""
        L.call("s2d_seed", self._use(), float(k0), float(amplitude), int(seed) & 0xFFFFFFFF)

    def seedPhysical(self, values):
        """solver.js:361-382: physical vorticity field of n*n floats."""
        v = np.ascontiguousarray(np.asarray(values, np.float32).reshape(-1))
        if v.size != self.ncells:
            raise ValueError(f"seedPhysical expects {self.ncells} values, got {v.size}")
        L.call("s2d_seed_physical", self._use(), _fptr(v))

    def seedBand(self, kmin: float, kmax: float, rms: float = 1.0, seed: int = 0):
        """Band-limited Gaussian initial spectrum of the benchmark workloads."""
        L.call("s2d_seed_band", self._use(), float(kmin), float(kmax), float(rms), int(seed) & 0xFFFFFFFF)

    def reset(self, opts: dict | None = None):
        """solver.js:420-444: ``{'field': ...}`` or ``{'k0', 'amplitude', 'seed', 'dyePattern'}``."""
        opts = opts or {}
        pattern = _PATTERNS[opts.get("dyePattern", "bands")]
        field = opts.get("field")
        if field is not None:
            v = np.ascontiguousarray(np.asarray(field, np.float32).reshape(-1))
            if v.size != self.ncells:
                raise ValueError(f"reset field expects {self.ncells} values, got {v.size}")
            L.call("s2d_reset", self._use(), _fptr(v), 0.0, 0.0, 0, pattern)
        else:
            L.call("s2d_reset", self._use(), None, float(opts.get("k0", 14)), float(opts.get("amplitude", 6)),
                   int(opts.get("seed", 1)) & 0xFFFFFFFF, pattern)

    def scenarioField(self, name: str, cfg: dict | None = None):
        """SCENARIOS[name].build(n, cfg) (scenarios.js) evaluated on the GPU: (n, n) float32."""
        from . import scenarios
        return scenarios.build(self, name, cfg)

    def resetScenario(self, name: str, cfg: dict | None = None, dyePattern: str = "bands"):
        """reset({field: SCENARIOS[name].build(n, cfg), dyePattern}) (main.js:281-283), the
        field built and seeded on the device."""
        from . import scenarios
        scenarios.reset(self, name, cfg, dyePattern)

    def autotune(self, steps: int = 20) -> dict:
        """Time every registered launch shape of the column and row stage kernels on this
        solver's state (restored afterwards) and keep the fastest (no reference counterpart).
        Returns {"column": [(shape, us per RK3 step), ...], "row": [...], "choice": {...}}."""
        rep = L.s2d_tune_report()
        L.call("s2d_autotune", self._use(), int(steps), C.byref(rep))

        def name(kind, i):
            buf = C.create_string_buffer(64)
            L.call("s2d_tune_variant_name", self._h, kind, i, buf, 64)
            return buf.value.decode()
        col = [(name(0, i), float(rep.phys_us[i])) for i in range(rep.phys_variants)]
        row = [(name(1, i), float(rep.spec_us[i])) for i in range(rep.spec_variants)]
        return {"column": col, "row": row,
                "choice": {"column": col[rep.phys_choice][0], "row": row[rep.spec_choice][0]}}

    def tuneVariantNames(self, kind: str = "row") -> list:
        """Names of the registered launch shapes of the column ("column") or row ("row")
        stage; for a tensor-core solver the last row shape is the row stage on the
        tensor cores."""
        k = 0 if kind == "column" else 1
        names = []
        buf = C.create_string_buffer(64)
        while L.lib().s2d_tune_variant_name(self._use(), k, len(names), buf, 64) == 0:
            names.append(buf.value.decode())
        return names

    def tuneSelect(self, column: int, row: int):
        """Use registered stage-kernel shapes `column` / `row` (indices of autotune's lists)."""
        L.call("s2d_tune_select", self._use(), int(column), int(row))

    def render(self, cfg: dict | None = None, width: int | None = None, height: int | None = None):
        """Renderer.render(encoder, solver, cfg) (render.js:63-87) without a canvas: an
        (height, width, 4) uint8 RGBA image, row 0 at the top.  cfg keys: mode (render.js:4
        names), exposure, vortScale, dyeGain; the image defaults to the dye grid's size."""
        cfg = cfg or {}
        mode = cfg.get("mode", "dye over vorticity")
        idx = L.RENDER_MODES.index(mode) if mode in L.RENDER_MODES else 0      # render.js:65
        w = self.m if width is None else int(width)
        h = self.m if height is None else int(height)
        out = np.empty((h, w, 4), np.uint8)
        L.call("s2d_render", self._use(), idx, float(cfg.get("exposure", 1.3)), float(cfg.get("vortScale", 0.16)),
               float(cfg.get("dyeGain", 1.0)), w, h, out.ctypes.data_as(C.c_void_p))
        return out

    def paintDye(self, pattern: str):
        """solver.js:446-473."""
        if pattern not in _PATTERNS:
            raise ValueError(f"unknown dye pattern {pattern!r}")
        L.call("s2d_paint_dye", self._use(), _PATTERNS[pattern])

    # ---------------------------------------------------------------- stepping
    def encodePrime(self, pass_=None):
        L.call("s2d_encode_prime", self._use())

    def encodeStep(self, pass_=None):
        L.call("s2d_encode_step", self._use())

    def encodeDye(self, pass_=None):
        L.call("s2d_encode_dye", self._use())

    def encodeDyePasses(self, pass_=None):
        """encodeDye as the reference's three dispatches (same bits as encodeDye)."""
        L.call("s2d_encode_dye_passes", self._use())

    def encodeReduce(self, pass_=None):
        L.call("s2d_encode_reduce", self._use())

    def step(self, substeps: int = 1, dye: bool = True, reduce: bool = True, graph: bool = False,
             relatch: bool = False):
        """The main.js:409-419 substep loop in one call (primes first when needed).

        ``relatch`` gives every substep its own stochastic-forcing phase, as a
        configure() before each substep would; ``graph`` replays a captured substep.
        """
        flags = ((L.S2D_STEP_DYE if dye else 0) | (L.S2D_STEP_REDUCE if reduce else 0)
                 | (L.S2D_STEP_RELATCH if relatch else 0))
        L.call("s2d_step_graph" if graph else "s2d_step", self._use(), int(substeps), flags)

    # ---------------------------------------------------------------- diagnostics
    def encodeDiagnostics(self, pass_=None):
        L.call("s2d_encode_diagnostics", self._use())

    def copyDiagnostics(self, encoder=None):
        L.call("s2d_copy_diagnostics", self._use())

    def pollDiagnostics(self) -> bool:
        return bool(L.check(L.lib().s2d_poll_diagnostics(self._use()), "s2d_poll_diagnostics"))

    def readDiagnostics(self):
        """solver.js:570-608: dict or None (nothing copied, or destroyed)."""
        if self.disposed:
            return None
        spec = np.zeros(self.nbins, np.float64)
        zonal = np.zeros(self.n, np.float32)
        e, z = C.c_double(), C.c_double()
        dt, sp = C.c_float(), C.c_float()
        st = L.call("s2d_read_diagnostics", self._h, spec.ctypes.data_as(C.POINTER(C.c_double)), _fptr(zonal),
                    C.byref(e), C.byref(z), C.byref(dt), C.byref(sp))
        if st == L.S2D_NO_DATA:
            return None
        return {"spectrum": spec, "zonal": zonal, "energy": e.value, "enstrophy": z.value,
                "dt": dt.value, "maxSpeed": sp.value}

    def readDiagnosticsFixed(self) -> dict:
        """The reference's u32 fixed-point decoding of the last copied diagnostics."""
        spec = np.zeros(self.nbins, np.float32)
        e, z = C.c_float(), C.c_float()
        L.call("s2d_read_diagnostics_fixed", self._use(), _fptr(spec), C.byref(e), C.byref(z))
        return {"spectrum": spec, "energy": e.value, "enstrophy": z.value}

    # ---------------------------------------------------------------- instrumentation
    PROFILE_CLASSES = ("phys_cols", "spec_rows", "dye", "force", "other")

    def profile(self, enable: bool):
        """Record CUDA events around every kernel launched by the non-graph calls."""
        L.call("s2d_profile", self._use(), 1 if enable else 0)

    def profileRead(self) -> dict:
        """{class: (device ms, launches)} since the last read (synchronizes)."""
        ms = (C.c_double * 5)()
        cnt = (C.c_int * 5)()
        L.call("s2d_profile_read", self._use(), ms, cnt)
        return {k: (ms[i], cnt[i]) for i, k in enumerate(self.PROFILE_CLASSES)}

    # ---------------------------------------------------------------- dye
    @property
    def currentDye(self) -> np.ndarray:
        """solver.js:610-612: the current dye texture as binary16 bits [m, m, 4]."""
        out = np.zeros((self.m, self.m, 4), np.uint16)
        L.call("s2d_get_dye", self._use(), out.ctypes.data_as(C.POINTER(C.c_uint16)))
        return out

    def setDye(self, bits):
        b = np.ascontiguousarray(np.asarray(bits, np.uint16).reshape(self.m, self.m, 4))
        L.call("s2d_set_dye", self._use(), b.ctypes.data_as(C.POINTER(C.c_uint16)))

    # ---------------------------------------------------------------- stage hooks (tests/index.html)
    def getBuffer(self, name: str) -> np.ndarray:
        bid = L.BUFFER_IDS[name]
        if name == "dt":
            out = np.zeros(4, np.float32)
            L.call("s2d_get_buffer", self._use(), bid, out.ctypes.data, out.nbytes)
            return out
        out = np.zeros((self.n, self.n), np.complex64)
        L.call("s2d_get_buffer", self._use(), bid, out.ctypes.data, out.nbytes)
        return out

    def setBuffer(self, name: str, values):
        bid = L.BUFFER_IDS[name]
        if name == "dt":
            a = np.ascontiguousarray(np.asarray(values, np.float32).reshape(-1))
        else:
            a = np.ascontiguousarray(np.asarray(values).astype(np.complex64).reshape(self.n, self.n))
        L.call("s2d_set_buffer", self._use(), bid, a.ctypes.data, a.nbytes)

    def velocityPack(self, stateIndex: int):
        L.call("s2d_velocity_pack", self._use(), int(stateIndex))

    def nlPack(self):
        L.call("s2d_nl_pack", self._use())

    def assemble(self):
        L.call("s2d_assemble", self._use())

    def rk3Stage(self, stage: int):
        L.call("s2d_rk3_stage", self._use(), int(stage))

    def encodeStepUnfused(self):
        """The reference's 33-dispatch encodeStep order (solver.js:488-521) built
        from the per-stage hooks; used to cross-check the fused step."""
        h = self._use()
        if self.cfg is None:
            raise RuntimeError("configure() first")
        self.setBuffer("force", np.zeros((self.n, self.n), np.complex64))
        p = self.phase
        for stage in range(3):
            self.velocityPack((p + stage) % 3)
            self.fft.inverse(None, "packA")
            self.fft.inverse(None, "packB")
            self.nlPack()
            self.fft.forward(None, "physZ")
            self.assemble()
            self.rk3Stage(stage)
        info = self._info()
        L.call("s2d_set_phase", h, (p + 1) % 3, info.dye_parity)
