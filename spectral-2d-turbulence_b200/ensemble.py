"""Host-side ``Ensemble``: many independent simulations of uneven grid sizes.

Each instance is a doubly periodic vorticity solver with its own size
(64..1024), Laplacian/hyper viscosity, beta, drag, forcing and fixed step;
every pass of an RK3 stage runs as one persistent launch over all of them, and
a step replays a captured CUDA graph.  The reference has no counterpart beyond
running several ``Solver`` objects side by side.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class Ensemble:
    def __init__(self, instances, device: int = 0):
        """``instances``: dicts with keys n, beta, drag, nuH, hyperP, dt and optional
        forceAmp, forceK, forceWidth, seed."""
        self.instances = [dict(i) for i in instances]
        arr = (L.s2d_instance_desc * len(self.instances))()
        for k, d in enumerate(self.instances):
            arr[k].n = int(d["n"])
            arr[k].beta = float(d.get("beta", 0.0))
            arr[k].drag = float(d.get("drag", 0.0))
            arr[k].nu_h = float(d.get("nuH", 0.0))
            arr[k].hyper_p = int(d.get("hyperP", 1))
            arr[k].dt = float(d["dt"])
            arr[k].force_amp = float(d.get("forceAmp", 0.0))
            arr[k].force_k = float(d.get("forceK", 0.0))
            arr[k].force_width = float(d.get("forceWidth", 1.0))
            arr[k].seed = int(d.get("seed", k)) & 0xFFFFFFFF
        h = C.c_void_p()
        L.call("s2d_ensemble_create", arr, len(self.instances), int(device), C.byref(h))
        self._h = h
        self.device = device

    @property
    def count(self) -> int:
        return len(self.instances)

    @property
    def stream(self) -> int:
        p = C.c_void_p()
        L.call("s2d_ensemble_get_stream", self._h, C.byref(p))
        return p.value or 0

    def seedBand(self, kmin: float, kmax: float, rms: float = 1.0):
        L.call("s2d_ensemble_seed_band", self._h, float(kmin), float(kmax), float(rms))

    def setState(self, index: int, spectrum):
        n = self.instances[index]["n"]
        a = np.ascontiguousarray(np.asarray(spectrum).astype(np.complex64).reshape(n, n))
        L.call("s2d_ensemble_set_state", self._h, int(index), a.ctypes.data_as(C.POINTER(C.c_float)))

    def getState(self, index: int) -> np.ndarray:
        n = self.instances[index]["n"]
        out = np.zeros((n, n), np.complex64)
        L.call("s2d_ensemble_get_state", self._h, int(index), out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def step(self, steps: int = 1, graph: bool = True):
        L.call("s2d_ensemble_step", self._h, int(steps), 1 if graph else 0)

    def autotune(self, steps: int = 3) -> dict:
        """Pick the resident-CTA shapes of the persistent stage kernels by timing them on
        this ensemble (state restored afterwards); no reference counterpart."""
        rep = L.s2d_tune_report()
        L.call("s2d_ensemble_autotune", self._h, int(steps), C.byref(rep))

        def name(kind, i):
            buf = C.create_string_buffer(64)
            L.call("s2d_ensemble_tune_variant_name", self._h, kind, i, buf, 64)
            return buf.value.decode()
        col = [(name(0, i), float(rep.phys_us[i])) for i in range(rep.phys_variants)]
        row = [(name(1, i), float(rep.spec_us[i])) for i in range(rep.spec_variants)]
        return {"column": col, "row": row,
                "choice": {"column": col[rep.phys_choice][0], "row": row[rep.spec_choice][0]}}

    def tuneSelect(self, column: int, row: int):
        """Pin the column / row shapes (indices into autotune()'s lists); no reference
        counterpart."""
        L.call("s2d_ensemble_tune_select", self._h, int(column), int(row))

    def synchronize(self):
        L.call("s2d_ensemble_synchronize", self._h)

    def energy(self):
        e = np.zeros(self.count, np.float64)
        z = np.zeros(self.count, np.float64)
        L.call("s2d_ensemble_energy", self._h, e.ctypes.data_as(C.POINTER(C.c_double)),
               z.ctypes.data_as(C.POINTER(C.c_double)))
        return e, z

    def destroy(self):
        if self._h is not None:
            L.call("s2d_ensemble_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
