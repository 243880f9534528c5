#!/usr/bin/env python
"""Benchmark of the integrating-factor RK3 pseudo-spectral step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the forced inverse-cascade configuration at 1024^2, FP32 FFT): one
benchmark step is one substep of the reference's frame loop, i.e. one RK3 step
(3 stages, 9 FFTs) + BFECC dye advection on the 2x refined 2048^2 dye grid +
the CFL reduction; white-in-time stochastic forcing in the annulus |k| = 64+-2
(amplitude 0.1), order-4 hyperviscosity with damping rate 1 at the dealias cutoff
(nu4 = 5.4e-21; the written nu4 = 1e-16 overflows the FP32 integrating factor at the
band corner), drag 1e-2, beta 0, CFL 0.5 capped at dt = 1e-3; seeded band-limited
initial field (4 <= |k| <= 12, rms vorticity 1).  Inputs are synthetic and generated
on the device.

Rank 0 prints ONE JSON line.  ``value`` is device-timed whole-job steps/s
(CUDA events on the solver stream, barrier + synchronize around the timed
region, max over ranks; N ranks run N independent replicas: "replicas only",
weak scaling).  ``e2e`` is the same metric through the public Solver API with
per-step host->device parameter/splat uploads (pinned host memory) and a
device->host diagnostics read inside the timed region; reads run one step behind,
as the reference's frame loop resolves its async readDiagnostics while the next
frame runs, and the last step's read is inside the timed region too.  ``roofline`` covers the dominant kernel,
``cpu_baseline`` the FP64 NumPy restatement of reference/spectral2d.py on the
host started from the GPU arm's own initial field, ``ensemble`` the batched 256 x 256^2 ensemble, ``ensemble_mixed`` the mixed batch
128 x 128^2 + 256 x 256^2 + 32 x 512^2.

``--impl reference`` times the reference's CPU algorithm (the oracle port of
reference/spectral2d.py, NumPy FP64) on the same workload with every host core
running one replica, and prints the same line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "RK3 steps/s (1024^2; 256x256^2 batch): TC split-FFT vs FP32 at rel err <=1e-5"
UNIT = "steps/s"
N = 1024
DYE_SCALE = 2
HYPER_P = 4
# Order-4 hyperviscosity given as the damping rate at the dealias cutoff, 1.0 (the
# reference's 'inverse cascade' preset, main.js:52-62): nu4 = 1/(N/3)^8 = 5.55e-21 at
# 1024^2.  The value 1e-16 of the written benchmark configuration puts
# E(-dt/2) = exp(+146) at the corner of the dealias band, beyond FP32 range: the
# reference's own integrating-factor RK3 (solver.wgsl:97-122) overflows there.
VISC_RATE = 1.0
NU4 = VISC_RATE / (N / 3.0) ** (2 * HYPER_P)
CFG = {"beta": 0.0, "drag": 1e-2, "viscosity": VISC_RATE, "hyperP": HYPER_P,
       "forceAmp": 0.1, "forceK": 64.0, "forceWidth": 2.0, "cfl": 0.5, "dtMin": 1e-6, "dtMax": 1e-3,
       "dyeFade": 0.999}
WORKLOAD = "forced inverse cascade 1024^2 FP32, dye 2048^2 (config 2 of the reference benchmark set)"
L2_BYTES = 126 * 2 ** 20


def _rows_in_band(n):
    kcut = n / 3.0
    return sum(1 for i in range(n) if abs(i if i < n // 2 else i - n) < kcut)


def algorithmic_bytes(n, m):
    """Per-launch algorithmic HBM bytes of each kernel class (averaged over the 3 stages)."""
    rb = _rows_in_band(n)
    c = 8 * n * n
    phys = 2 * c + 8 * n * rb + c / 3.0                  # PA+PB read, in-band Z rows written, vel at stage 2
    spec = 8 * n * rb + 4 * c + 2 * c / 3.0              # Z rows, wcur, wout, PA, PB; w0 at stages 1-2
    dye = 16 * m * m + 8 * n * n                         # one dye texture read + one written, velocity read
    return {"phys_cols": phys, "spec_rows": spec, "dye": dye}


def step_algorithmic_bytes(n):
    """Minimum-pass dataflow of one RK3 step, 232 N^2 bytes (dye and pointer forcing excluded)."""
    return 232 * n * n


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), float(d.get("bf16_tflops", 1590.0)), "measured"
    return 6650.0, 1590.0, "fallback"


def committed_traffic(kernel):
    """DRAM bytes per launch of `kernel` recorded from an ncu capture under profiles/."""
    pat = re.compile(r"^traffic_bytes_per_launch\s+(\S+)\s+([0-9.eE+]+)")
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if not f.endswith((".md", ".txt")):
            continue
        with open(os.path.join(d, f)) as fh:
            for line in fh:
                m = pat.match(line.strip())
                if m and m.group(1) == kernel:
                    return float(m.group(2))
    return None


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    NVML is polled every 2 ms on a thread (the timed region can be tens of
    milliseconds, shorter than nvidia-smi's own sampling start-up); only samples
    taken between mark_start() and mark_end() count.  nvidia-smi -lms 100 is the
    fallback when NVML is unavailable.  Read-only: no setting of the GPU changes.
    """
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []            # (time, sm_mhz, reasons bitmask)
        self.smax = None
        self.t0 = self.t1 = None
        self.stop_flag = threading.Event()
        self.nvml = None
        self.proc = None
        self.lines = []

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.gpu)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            self.nvml, self.h = self._nvml_handle()
            self.smax = float(self.nvml.nvmlDeviceGetMaxClockInfo(self.h, self.nvml.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _poll(self):
        nv, h = self.nvml, self.h
        while not self.stop_flag.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((time.perf_counter(), mhz, rs))
            except Exception:
                pass
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()

    def _in_window(self, t):
        return (self.t0 is None or t >= self.t0) and (self.t1 is None or t <= self.t1)

    def stop(self):
        self.stop_flag.set()
        sm, reasons = [], set()
        if self.nvml is not None:
            self.thread.join(timeout=2)
            for t, mhz, rs in self.samples:
                if not self._in_window(t):
                    continue
                sm.append(mhz)
                for nm, bit in self.REASONS:
                    if rs & bit:
                        reasons.add(nm)
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 2 ms polling"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        smax = None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9 or not self._in_window(t):
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi -lms 100"}


# ------------------------------------------------------------------ distributed plumbing
def dist_setup(gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([float(x)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_by_cost(instances, world):
    """Split ensemble instances over `world` ranks with balanced cost N^2 log2 N (greedy,
    largest first into the least-loaded rank; ties to the lower rank) -- deterministic, so
    every rank computes the same partition without communicating."""
    import math
    order = sorted(range(len(instances)), key=lambda i: (-instances[i]["n"], i))
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        n = instances[i]["n"]
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(instances[i])
        load[r] += n * n * math.log2(n)
    return shards


# ------------------------------------------------------------------ CPU reference arm
def _oracle_worker(args):
    """Run `steps` oracle steps of the workload -- an RK3 step with forcing and the CFL dt,
    then the BFECC dye step on the (N * DYE_SCALE)^2 dye with that step's velocity, as the
    GPU arm's step does -- and return (steps, seconds).

    The initial field is `w0` when given (the GPU arm's own initial state, read back from
    the device), else the CPU restatement of the device band seed s2d_seed_band with the
    GPU arm's seed (1 + rank), so both arms start from the same FP32 field; the dye starts
    as the 'bands' pattern, as the GPU arm's reset paints it."""
    n, steps, seed, w0 = args
    import numpy as np
    from oracle import wgsl_oracle as wo
    from oracle.spectral_oracle import SpectralOracle
    nu_h = float(wo.nu_h_from_rate(CFG["viscosity"], n, HYPER_P))
    s = SpectralOracle(n=n, beta=CFG["beta"], mu=CFG["drag"], nu_h=nu_h, hyper_p=HYPER_P, cfl=CFG["cfl"],
                       dt_max=CFG["dtMax"])
    init = w0 if w0 is not None else wo.band_seed_spectrum(n, 4.0, 12.0, 1.0, seed)
    s.w = np.asarray(init).astype(np.complex128)
    s.step(dt=CFG["dtMax"])        # warm-up
    s.w = np.asarray(init).astype(np.complex128)
    dye = wo.paint_dye_bands(n * DYE_SCALE)
    t0 = time.perf_counter()
    for k in range(steps):
        dt = s.timestep()
        f = wo.stochastic_forcing(n, CFG["forceAmp"], CFG["forceK"], CFG["forceWidth"], k, dt)
        s.step(dt=dt, forcing=f.astype(np.complex128))
        u, v = s.velocity()
        dye = wo.dye_step(dye, np.stack([u, v], axis=-1).astype(np.float32), dt, CFG["dyeFade"])
    return steps, time.perf_counter() - t0


def cpu_baseline(w0, budget_s=15.0):
    """The FP64 NumPy restatement of reference/spectral2d.py plus the FP32 restatement of
    the dye shader, one core, bounded sample, started from the GPU arm's own initial field
    `w0` (the same FP32 bits)."""
    steps1, t1 = _oracle_worker((N, 1, 1, w0))
    k = max(1, min(20, int(budget_s / max(t1, 1e-3))))
    steps, secs = _oracle_worker((N, k, 1, w0))
    return {"value": steps / secs, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{steps} steps of one {N}^2 instance: RK3 with forcing and CFL dt (FP64 NumPy "
                      f"restatement of reference/spectral2d.py) and the BFECC dye step on the "
                      f"{N * DYE_SCALE}^2 dye (NumPy restatement of dye.wgsl), {secs:.1f} s; initial field = "
                      "the GPU arm's seeded state read back from the device (same FP32 bits)"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    procs = max(1, min(os.cpu_count() or 1, 16))
    # bound the run: each replica does at most what fits ~90 s of host time
    _, t1 = _oracle_worker((N, 1, 1, None))
    per = max(1, min(args.steps, int(90.0 / max(t1, 1e-3))))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_oracle_worker, [(N, per, 1 + r, None) for r in range(procs)])
    wall = time.perf_counter() - t0
    steps = sum(r[0] for r in res)
    secs = max(r[1] for r in res)
    value = steps / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / per,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": N, "dye": N * DYE_SCALE, "replicas": procs},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                         "sample": f"{procs} processes x {per} steps at {N}^2, each an RK3 step (NumPy FP64 "
                                   f"restatement of reference/spectral2d.py) and a BFECC dye step on the "
                                   f"{N * DYE_SCALE}^2 dye (NumPy restatement of dye.wgsl); wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def run_ours(args):
    import torch
    world, rank, local = dist_setup(args.gpus)
    import __graft_entry__ as ge
    pkg = ge.load_package()
    dev = local
    torch.cuda.set_device(dev)

    solver = pkg.Solver.create(device=dev, n=N, dyeScale=DYE_SCALE)
    solver.configure(CFG)
    solver.reset({"k0": 14, "amplitude": 0, "seed": 1, "dyePattern": "bands"})
    solver.seedBand(4.0, 12.0, rms=1.0, seed=1 + rank)
    w_init = solver.getBuffer("state0") if (rank == 0 and world == 1 and not args.no_cpu) else None
    stream = torch.cuda.ExternalStream(solver.stream, device=dev)
    # stage-kernel launch shapes chosen by the library's autotuner (before any timing), or
    # pinned with --shapes (reproducible profiling)
    tune = pinned_shapes(solver, args.shapes) if args.shapes else solver.autotune(20)

    # warm-up (also captures the graphs of the 6 (phase, dt slot, dye parity) combinations)
    solver.step(max(args.warmup, 6), dye=True, reduce=True, graph=True, relatch=True)
    solver.synchronize()

    # ---- device-timed region
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.05)                      # the poller is running before the timed region
    barrier(world)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark_start()
    ev0.record(stream)
    solver.step(args.steps, dye=True, reduce=True, graph=True, relatch=True)
    ev1.record(stream)
    ev1.synchronize()
    clocks.mark_end()
    torch.cuda.synchronize(dev)
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, world)
    value = world * args.steps / (ms / 1e3)

    # ---- RK3-only (no dye) for reference
    solver.step(3, dye=False, reduce=True, graph=True, relatch=True)
    solver.synchronize()
    ev0.record(stream)
    solver.step(args.steps, dye=False, reduce=True, graph=True, relatch=True)
    ev1.record(stream)
    ev1.synchronize()
    ms_rk3 = max_over_ranks(ev0.elapsed_time(ev1), world)

    # ---- per-kernel device times: event-record nodes around each kernel class inside the
    # replayed graphs (each replay synchronized and read, so no host gaps are timed)
    ksteps = min(args.steps, 60)
    solver.profile(True)
    solver.step(6, dye=True, reduce=True, graph=True, relatch=True)     # capture the profiled graphs
    solver.profileRead()
    solver.step(ksteps, dye=True, reduce=True, graph=True, relatch=True)
    prof = solver.profileRead()
    if not any(prof[k][1] for k in ("phys_cols", "spec_rows", "dye")):
        # event nodes unreadable in this driver: time the same steps launch by launch
        solver.step(ksteps, dye=True, reduce=True, graph=False, relatch=True)
        prof = solver.profileRead()
    solver.profile(False)
    ab = algorithmic_bytes(N, N * DYE_SCALE)
    hbm, bf16, peak_src = load_peaks()
    dom = max(("phys_cols", "spec_rows", "dye"), key=lambda k: prof[k][0])
    dom_ms, dom_n = prof[dom]
    avg_launch_s = dom_ms / 1e3 / max(dom_n, 1)
    achieved = ab[dom] / avg_launch_s / 1e9
    kernel_names = {"phys_cols": "k_phys_cols", "spec_rows": "k_spec_rows", "dye": "k_dye_fused"}
    traffic = committed_traffic(kernel_names[dom].split()[0])
    step_ms = ms / args.steps if world == 1 else ms / args.steps
    roofline = {"bound": "hbm", "kernel": kernel_names[dom], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": ab[dom], "avg_launch_ms": avg_launch_s * 1e3,
                "per_kernel_ms_per_step": {k: prof[k][0] / ksteps for k in prof}}
    step_roof = step_algorithmic_bytes(N) / ((ms_rk3 / args.steps) / 1e3) / 1e9

    # ---- end to end through the public API: per step configure + splats + step + diagnostics
    # read.  Reads run one step behind, as the reference app's frame loop does (its
    # readDiagnostics is an async buffer map that resolves while the next frame runs): step k
    # is queued before the host waits for step k-1's copy, so the device never idles on the
    # host.  Every step's diagnostics are read; the last one before the clock stops.
    e2e_steps = min(max(args.steps, 100), 200)
    for _ in range(3):
        solver.configure(CFG)
        solver.setSplats([])
        solver.step(1, dye=True, reduce=True, graph=True)
        solver.encodeDiagnostics()
        solver.copyDiagnostics()
        solver.readDiagnostics()
    barrier(world)
    t0 = time.perf_counter()
    reads = 0
    for _ in range(e2e_steps):
        solver.configure(CFG)                       # H2D (pinned ring): parameter block
        solver.setSplats([])                        # H2D (pinned ring): splat block
        solver.step(1, dye=True, reduce=True, graph=True)
        solver.encodeDiagnostics()
        d = solver.readDiagnostics()                # D2H of step k-1: spectrum, zonal, dt, energies
        reads += d is not None
        solver.copyDiagnostics()                    # step k's copy, read next iteration
    d = solver.readDiagnostics()
    reads += d is not None
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    assert reads == e2e_steps, (reads, e2e_steps)
    e2e_value = world * e2e_steps / e2e_s
    nb = N // 2 + 1
    h2d = 64 + 16 + 8 * 48
    # two copies per step on the diagnostics stream: a diagnostics block (FP64 bins + u32
    # bins (+ totals), the zonal mean) and the current [dt, speed] slot
    d2h = (nb + 2) * 8 + (nb + 2) * 4 + N * 4 + 2 * 4
    finite = d is not None and all(map(lambda v: v == v, [d["energy"], d["enstrophy"], d["dt"]]))
    solver.destroy()

    # ---- the same step with the tensor-core (split FP16 DFT-GEMM) column stage
    tc = None
    if not args.no_tc:
        tc = run_tc_leg(pkg, torch, world, rank, dev, args, value, world * args.steps / (ms_rk3 / 1e3))

    # ---- batched ensemble: 256 instances of 256^2 (sharded across ranks)
    ens = ens_mixed = None
    if not args.no_ensemble:
        ens = run_ensemble(pkg, torch, world, rank, dev, args)
        ens_mixed = run_ensemble(pkg, torch, world, rank, dev, args, groups=ENSEMBLE_MIXED, seed=4321)

    cpu = cpu_baseline(w_init) if w_init is not None else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": N, "dye": N * DYE_SCALE, "fft": "fp32 CUDA-core",
                       "parallelism": f"replicas x{world}", "graph": True,
                       "l2": f"no flush; per-step working set {working_set(N, N * DYE_SCALE) / 2**20:.0f} MiB "
                             f"> L2 {L2_BYTES / 2**20:.0f} MiB",
                       "forcing": "white-in-time, |k|=64+-2, amp 0.1", "dt": "CFL 0.5, max 1e-3",
                       "hyperviscosity": f"p=4, nu4={NU4:.3g} (rate {VISC_RATE} at the cutoff)",
                       "drag": 1e-2, "autotune": tune},
            "rk3_only_steps_per_s": world * args.steps / (ms_rk3 / 1e3),
            "step_roofline": {"bytes_per_step": step_algorithmic_bytes(N), "achieved_gbs": step_roof,
                              "frac": step_roof / hbm, "note": "232 N^2 algorithmic bytes per RK3 step (no dye)"},
            "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "diagnostics_finite": bool(finite)},
            # per timed step: 3 k_phys_cols + 3 k_spec_rows + k_dye_fused (the CFL reduction
            # and the stepIndex latch are fused into k_phys_cols)
            "gpu_launches": args.steps * 7,
            "clocks": clk,
            "cpu_baseline": cpu,
            "tc_vs_fp32": tc,
            "ensemble": ens,
            "ensemble_mixed": ens_mixed,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def pinned_shapes(solver, spec):
    """--shapes C,R: use column shape C and row shape R (indices of Solver.autotune()'s lists)."""
    c, r = (int(v) for v in spec.split(","))
    solver.tuneSelect(c, r)
    return {"pinned": {"column": c, "row": r}}


def _timed_steps(solver, stream, torch, steps, dye):
    solver.step(3, dye=dye, reduce=True, graph=True, relatch=True)
    solver.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    solver.step(steps, dye=dye, reduce=True, graph=True, relatch=True)
    ev1.record(stream)
    ev1.synchronize()
    return ev0.elapsed_time(ev1)


def _bench_solver(pkg, dev, fft, seed):
    s = pkg.Solver.create(device=dev, n=N, dyeScale=DYE_SCALE, fft=fft)
    s.configure(CFG)
    s.reset({"k0": 14, "amplitude": 0, "seed": 1, "dyePattern": "bands"})
    s.seedBand(4.0, 12.0, rms=1.0, seed=seed)
    return s


def tc_divergence(pkg, dev, steps=10, fft_tc="tc-f16"):
    """rel L2 between the FP32 and a tensor-core step after 1 and `steps` steps of the
    benchmark configuration from the same seeded state (adaptive dt, forcing on)."""
    import numpy as np
    out = {}
    for fft in ("fp32", fft_tc):
        s = _bench_solver(pkg, dev, fft, 1)
        try:
            s.step(1, dye=False, reduce=True, graph=False)
            one = s.getBuffer(f"state{s.phase}")
            s.step(steps - 1, dye=False, reduce=True, graph=False)
            many = s.getBuffer(f"state{s.phase}")
            out[fft] = (one.astype(np.complex128), many.astype(np.complex128))
        finally:
            s.destroy()

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return {"1_step": rel(out[fft_tc][0], out["fp32"][0]),
            f"{steps}_steps": rel(out[fft_tc][1], out["fp32"][1])}


def run_tc_leg(pkg, torch, world, rank, dev, args, fp32_value, fp32_rk3):
    """Time the benchmark step with fft='tc-f16' (both y-transforms of every RK stage as
    split-FP16 tcgen05 DFT-GEMMs) exactly like the FP32 step, and measure how far it
    drifts from the FP32 step."""
    solver = _bench_solver(pkg, dev, "tc-f16", 1 + rank)
    stream = torch.cuda.ExternalStream(solver.stream, device=dev)
    tune = pinned_shapes(solver, args.shapes) if args.shapes else solver.autotune(20)
    solver.step(max(args.warmup, 6), dye=True, reduce=True, graph=True, relatch=True)
    solver.synchronize()
    barrier(world)
    ms = max_over_ranks(_timed_steps(solver, stream, torch, args.steps, True), world)
    ms_rk3 = max_over_ranks(_timed_steps(solver, stream, torch, args.steps, False), world)
    ksteps = min(args.steps, 60)
    solver.profile(True)
    solver.step(6, dye=False, reduce=True, graph=True, relatch=True)
    solver.profileRead()
    solver.step(ksteps, dye=False, reduce=True, graph=True, relatch=True)
    prof = solver.profileRead()
    solver.profile(False)
    solver.destroy()
    value = world * args.steps / (ms / 1e3)
    rk3 = world * args.steps / (ms_rk3 / 1e3)
    # the BF16 split (16 significant bits per operand): speed and drift from FP32
    bsolver = _bench_solver(pkg, dev, "tc-bf16", 1 + rank)
    bstream = torch.cuda.ExternalStream(bsolver.stream, device=dev)
    if args.shapes:
        pinned_shapes(bsolver, args.shapes)
    else:
        bsolver.autotune(5)
    bsolver.step(max(args.warmup, 6), dye=False, reduce=True, graph=True, relatch=True)
    bsolver.synchronize()
    ms_bf16 = max_over_ranks(_timed_steps(bsolver, bstream, torch, args.steps, False), world)
    bsolver.destroy()
    bf16 = {"rk3_only_steps_per_s": world * args.steps / (ms_bf16 / 1e3),
            "rel_l2_vs_fp32": tc_divergence(pkg, dev, fft_tc="tc-bf16")}
    return {"fft": "split FP16 hi+lo tcgen05 DFT-GEMM (y-transforms); FP32 row transforms",
            "bf16_split": bf16,
            "steps_per_s": value, "rk3_only_steps_per_s": rk3,
            "fp32_steps_per_s": fp32_value, "fp32_rk3_only_steps_per_s": fp32_rk3,
            "rk3_speedup_vs_fp32": rk3 / fp32_rk3, "speedup_vs_fp32": value / fp32_value,
            "per_kernel_ms_per_step": {k: prof[k][0] / ksteps for k in prof},
            "autotune": tune, "rel_l2_vs_fp32": tc_divergence(pkg, dev)}


def working_set(n, m):
    return 8 * n * n * 7 + 8 * m * m * 3


ENSEMBLE_256 = ((256, 256),)
# the mixed batch of the reference's ensemble configuration: 128 x 128^2, 256 x 256^2, 32 x 512^2
ENSEMBLE_MIXED = ((128, 128), (256, 256), (512, 32))


def run_ensemble(pkg, torch, world, rank, dev, args, groups=ENSEMBLE_256, seed=1234):
    """Graph-replayed RK3 steps of a batch of independent instances (sizes `groups` =
    (n, count) pairs), per-instance nu ~ U[1e-4, 1e-3], beta ~ U[0, 20], drag ~ U[0, 2e-2],
    band-limited initial fields; instances sharded by cost (N^2 log2 N, shard_by_cost) across ranks."""
    import numpy as np
    rng = np.random.default_rng(seed)
    inst = []
    for n, count in groups:
        for _ in range(count):
            inst.append({"n": n, "beta": float(rng.uniform(0, 20)), "drag": float(rng.uniform(0, 2e-2)),
                         "nuH": float(rng.uniform(1e-4, 1e-3)), "hyperP": 1, "dt": 2e-3, "seed": len(inst)})
    count_total = len(inst)
    mine = shard_by_cost(inst, world)[rank]
    e = pkg.Ensemble(mine, device=dev)
    e.seedBand(4.0, 12.0, rms=1.0)
    tune = e.autotune(3)                  # persistent-kernel shapes (state restored)
    stream = torch.cuda.ExternalStream(e.stream, device=dev)
    e.step(6, graph=True)
    e.synchronize()
    steps = max(3, (min(args.steps, 300) // 3) * 3)
    barrier(world)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    e.step(steps, graph=True)
    ev1.record(stream)
    ev1.synchronize()
    barrier(world)
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    en, _ = e.energy()
    ok = bool(np.all(np.isfinite(en)))
    e.destroy()
    hbm, _, _ = load_peaks()
    ens_steps_per_s = steps / (ms / 1e3)
    bytes_step = sum(step_algorithmic_bytes(n) * c for n, c in groups)
    gbs = bytes_step * ens_steps_per_s / 1e9
    out = {"instances": count_total, "sizes": {str(n): c for n, c in groups},
           "n": groups[0][0] if len(groups) == 1 else None, "ensemble_steps_per_s": ens_steps_per_s,
           "instance_steps_per_s": ens_steps_per_s * count_total, "ms_per_ensemble_step": ms / steps,
           "achieved_gbs": gbs, "hbm_peak_gbs": hbm, "frac_of_hbm": gbs / hbm, "finite": ok, "autotune": tune,
           "note": "232 N^2 algorithmic bytes per instance-step; per-instance nu, beta, drag; graph-replayed"}
    # the DRAM bytes the kernels actually move (ncu, committed under profiles/; recorded
    # for the 256 x 256^2 ensemble): the stage kernels skip out-of-band pack rows, so
    # they move fewer bytes than the algorithmic count, and this fraction is the one
    # that says how close to the bandwidth bound they run
    spec_b, phys_b = committed_traffic("k_ens_spec"), committed_traffic("k_ens_phys")
    if spec_b and phys_b and tuple(groups) == ENSEMBLE_256:
        moved = 3 * (spec_b + phys_b)
        out["dram_traffic"] = {"bytes_per_ensemble_step": moved, "gbs": moved * ens_steps_per_s / 1e9,
                               "frac_of_hbm": moved * ens_steps_per_s / 1e9 / hbm,
                               "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch"}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tc", action="store_true")
    ap.add_argument("--shapes", default=None,
                    help="C,R: pin the stage-kernel shapes (column C, row R) instead of autotuning")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
