/*
 * s2d.h -- C ABI of the B200 pseudo-spectral vorticity solver.
 *
 * This is the drop-in boundary for the reference's JavaScript solver API
 * (src/gpu/solver.js `class Solver`, src/gpu/fft.js `Fft2D`/`radixSchedule`,
 * src/gpu/device.js `supportedGrids`).  Each entry point names the reference
 * interface it replaces (file:line).  Plain C types only: pointers, sizes,
 * ints and floats.  Every call returns an int status (S2D_OK = 0, errors < 0);
 * the N-API / ctypes shims turn a negative status into a thrown Error with the
 * text of s2d_last_error().
 *
 * Data layout (identical to the reference buffers): a spectral field is N*N
 * interleaved complex64 (re, im float pairs), row-major, row = y index with
 * ky = wn(row), column = x index with kx = wn(col), wn(i) = i < N/2 ? i : i-N.
 * The dye is M*M texels of 4 binary16 values (rgba16float), M = N*dye_scale.
 *
 * Threading: a solver handle is used from one host thread at a time (except
 * s2d_poll_diagnostics, host-only, which another thread may call); the GPU work of
 * one solver runs on the solver's own CUDA stream, except the diagnostics spectra
 * and readback copies, which run on a second stream of the solver and are ordered
 * against the first by the library (s2d_encode_diagnostics).
 */
#ifndef S2D_H
#define S2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define S2D_OK 0
#define S2D_NO_DATA 1             /* readDiagnostics resolved to null (solver.js:571-573) */
#define S2D_ERR_ARG (-1)          /* bad argument / null handle                              */
#define S2D_ERR_UNSUPPORTED_N (-2)/* grid size not supported (fft.js:27-29)                 */
#define S2D_ERR_CUDA (-3)         /* CUDA runtime error (text in s2d_last_error)             */
#define S2D_ERR_DESTROYED (-4)    /* use after destroy (solver.js:571, 614-615)              */
#define S2D_ERR_NAN (-5)          /* non-finite value found in a host-provided field         */
#define S2D_ERR_UNREGISTERED (-6) /* FFT on a buffer never registered (fft.js:84)            */
#define S2D_ERR_NO_DEVICE (-7)    /* no CUDA device / wrong architecture                     */

/* ---------------------------------------------------------------- limits */
#define S2D_MAX_SPLATS 8          /* MAX_SPLATS, solver.js:9 */
#define S2D_MIN_N 32
#define S2D_MAX_N 4096

/* buffer ids of the per-stage test hooks (tests/index.html:120-201 names) */
enum s2d_buffer_id {
  S2D_BUF_STATE0 = 0, S2D_BUF_STATE1 = 1, S2D_BUF_STATE2 = 2,
  S2D_BUF_PACKA = 3, S2D_BUF_PACKB = 4, S2D_BUF_PHYSZ = 5,
  S2D_BUF_RHS = 6, S2D_BUF_FORCE = 7,
  S2D_BUF_VEL = 8,      /* N*N float2 (u, v), physical space */
  S2D_BUF_DT = 9        /* 4 floats: [dt, maxSpeed, 0, 0] of the current dt slot */
};

/* step flags: one substep of the main.js:413-419 loop is
 * encodeStep, then encodeDye, then encodeReduce */
#define S2D_STEP_DYE 1u
#define S2D_STEP_REDUCE 2u
/* Re-latch the stochastic-forcing step index before every substep, as a
 * configure() call before each substep would (main.js:403 calls configure once
 * per frame, so with one substep per frame every step gets a fresh phase). */
#define S2D_STEP_RELATCH 4u

/* FFT arithmetic of the fused step */
#define S2D_FFT_FP32 0            /* CUDA-core FP32 FFT */
/* Tensor-core DFT-GEMM FFT with split hi+lo operands and FP32 accumulation, N = 256, 512,
 * 1024, 2048, 4096 (other N: S2D_ERR_UNSUPPORTED_N).  At N = 1024 the step's stages are
 * fused tensor-core kernels; at the other sizes the step runs the reference's per-stage
 * order with every 2D transform on the tensor cores. */
#define S2D_FFT_TC_F16 1          /* FP16 hi+lo: 22 significant bits per operand */
#define S2D_FFT_TC_BF16 2         /* BF16 hi+lo: 16 significant bits per operand */

/* dye patterns of paintDye (solver.js:446-473) */
#define S2D_DYE_NONE 0
#define S2D_DYE_BANDS 1

/* Solver.configure(cfg) keys (solver.js:306-324).  `viscosity` is the damping
 * RATE at the dealias cutoff; nuH = viscosity / (N/3)^(2*hyperP) (solver.js:311). */
typedef struct s2d_params {
  float beta, drag, viscosity;
  int32_t hyper_p;
  float force_amp, force_k, force_width;
  float cfl, dt_min, dt_max;
  float dye_fade;
} s2d_params;

/* setSplats list entry (solver.js:326-345; built by ui/pointer.js:57-67).
 * x, y in [0,1)^2; (dx, dy) the stroke velocity; colour in [0,1]. */
typedef struct s2d_splat {
  float x, y, dx, dy;
  float color[3];
  float radius, amp, dye_amp;
} s2d_splat;

/* scalar state fields of the JS Solver (solver.js:50-69) */
typedef struct s2d_info {
  int32_t n, m, nbins;
  int32_t phase, dye_parity;
  uint32_t step_index;
  int32_t primed;
  int32_t fft_precision;
  float nu_h;           /* paramsF[2] */
  double sim_time;
} s2d_info;

typedef struct s2d_solver s2d_solver;

/* ---------------------------------------------------------------- library */
int s2d_version(void);
const char* s2d_status_string(int status);
const char* s2d_last_error(void);

/* radixSchedule(n) (fft.js:20-31): stages of radix 4 and whether a radix-2 tail
 * is present; S2D_ERR_UNSUPPORTED_N for n not of the form 4^a or 2*4^a. */
int s2d_radix_schedule(int n, int* stages, int* has_radix2);
/* supportedGrids(limits) (device.js:44-52), re-derived for the current B200:
 * writes the supported sizes in [S2D_MIN_N, S2D_MAX_N] ascending. */
int s2d_supported_grids(int* out, int capacity, int* count);
/* Bit-exact tables computed by GPU kernels (for parity tests):
 * digit reversal over the reversed radix list (fft.wgsl:32-40, fft_ref.py:19-24),
 * wn(i) as float (common.wgsl:50-55), and the 2/3 dealias mask (common.wgsl:69-74). */
int s2d_digit_reverse_table(int n, uint32_t* out /* n */);
int s2d_wavenumber_table(int n, float* out /* n */);
int s2d_dealias_mask_table(int n, uint8_t* out /* n*n */);
/* Self-check of the fused dye kernel's tile geometry (no reference counterpart; host
 * only, no GPU needed): for an n x n flow under an (n * dye_scale)^2 dye, every tile's
 * traces shorter than one texel -- the tiles that skip the window bounds tests -- read
 * only velocity cells inside the tile's velocity window and only dye texels inside the
 * tile's source / forward / backward windows.  S2D_OK, or S2D_ERR_ARG naming the first
 * tile and window that would be left. */
int s2d_dye_fast_path_check(int n, int dye_scale);

/* ---------------------------------------------------------------- lifecycle */
/* Solver.create(device, {n, dyeScale}) (solver.js:71-140).  dye_scale is 1, 2 (the
 * reference's two choices, main.js:196) or 4; any other value is S2D_ERR_ARG. */
int s2d_create(int n, int dye_scale, int fft_precision, int device, s2d_solver** out);
/* Solver.destroy() (solver.js:614-629); the handle is freed. */
int s2d_destroy(s2d_solver* s);
int s2d_get_info(s2d_solver* s, s2d_info* out);
/* solver.phase / dyeParity / simTime assignments made by tests/index.html:162,185-186 */
int s2d_set_phase(s2d_solver* s, int phase, int dye_parity);
int s2d_set_sim_time(s2d_solver* s, double t);
/* CUDA stream the solver enqueues on (cudaStream_t as void*), created at the highest
 * stream priority.  The diagnostics spectra and readback copies run on a second,
 * lowest-priority stream of the solver (see s2d_encode_diagnostics). */
int s2d_get_stream(s2d_solver* s, void** stream);
/* Waits for both streams and reports a bounded device-side wait that gave up. */
int s2d_synchronize(s2d_solver* s);
/* Failure-detection check (no reference counterpart; the reference's WebGPU queue has no
 * device-side waits).  Every device-side wait of the library (bulk-copy and MMA
 * barriers) gives up after a global-timer limit (50 ms), records its site in the
 * solver's error word and lets the kernel return; the next s2d_synchronize (or any call
 * that reads the word) returns S2D_ERR_CUDA.  This enqueues one CTA whose wait can
 * never complete (its barrier expects bytes that are never sent), with a limit of
 * limit_ns (1..1e9), so that path can be exercised without faulting the GPU. */
int s2d_probe_wait_timeout(s2d_solver* s, unsigned long long limit_ns);

/* ---------------------------------------------------------------- parameters */
/* Both update the solver's host copy of the parameter / splat block and return; the
 * blocks that changed reach the device together, in one copy from pinned memory, at the
 * start of the next call that enqueues device work or reads the device (every s2d_*
 * call on the solver except these two, s2d_get_info, s2d_set_phase, s2d_set_sim_time,
 * s2d_get_stream and s2d_poll_diagnostics) -- in stream order before that call's work, as the reference's
 * writeBuffer precedes the passes encoded after it.  Work a caller enqueues on the
 * solver's stream directly sees the blocks after the next such call. */
int s2d_configure(s2d_solver* s, const s2d_params* p);                   /* solver.js:306-324 */
int s2d_set_splats(s2d_solver* s, const s2d_splat* list, int count);     /* solver.js:326-345 */

/* ---------------------------------------------------------------- seeding */
/* seed({k0, amplitude, seed}) (solver.js:347-359, fillSpectrum 384-418). */
int s2d_seed(s2d_solver* s, double k0, double amplitude, uint32_t seed);
/* seedPhysical(Float32Array N*N) (solver.js:361-382): FFT + dealias mask into state 0. */
int s2d_seed_physical(s2d_solver* s, const float* field);
/* reset({field} | {k0, amplitude, seed, dyePattern}) (solver.js:420-444);
 * field == NULL selects spectral seeding. */
int s2d_reset(s2d_solver* s, const float* field, double k0, double amplitude, uint32_t seed,
              int dye_pattern);
int s2d_paint_dye(s2d_solver* s, int pattern);                           /* solver.js:446-473 */
/* Band-limited initial spectrum of the benchmark workloads: complex Gaussian
 * noise (counter-based, from `seed`) kept in kmin <= |k| <= kmax,
 * Hermitian-symmetrised, dealias-masked, k=0 removed, scaled to rms vorticity
 * `rms`; into state 0 with the other states cleared.  No reference
 * counterpart (the reference seeds with fillSpectrum or a physical field). */
int s2d_seed_band(s2d_solver* s, float kmin, float kmax, float rms, uint32_t seed);

/* Scenario initial fields (scenarios.js:3-163, SCENARIOS).  `param` is
 * cfg.mergerSep for MERGER (scenarios.js:137) and cfg.polygonN for POLYGON
 * (scenarios.js:158, rounded, 1..S2D_SCENARIO_MAX_BLOBS), ignored otherwise.
 * The field is evaluated on the device in FP64 and rounded to FP32, as the
 * reference's Float32Array holds it. */
#define S2D_SCENARIO_SHEAR_LAYER 0
#define S2D_SCENARIO_TAYLOR_GREEN 1
#define S2D_SCENARIO_DIPOLE 2
#define S2D_SCENARIO_MERGER 3
#define S2D_SCENARIO_POLYGON 4
#define S2D_SCENARIO_MAX_BLOBS 256
/* SCENARIOS[kind].build(n, cfg) (scenarios.js) into host memory, n*n floats row-major */
int s2d_scenario_field(s2d_solver* s, int kind, double param, float* field_out);
/* reset({field: SCENARIOS[kind].build(n, cfg), dyePattern}) (main.js:281-283 with
 * solver.js:420-444), the field never leaving the device */
int s2d_reset_scenario(s2d_solver* s, int kind, double param, int dye_pattern);

/* ---------------------------------------------------------------- autotuner */
/* No counterpart in the reference (its kernels have one fixed shape).  Each grid
 * size registers up to S2D_TUNE_MAX launch shapes of the column and the row stage
 * kernels (values per thread / radix of the line passes, resident CTAs per SM);
 * s2d_autotune times them on this solver's own state (`steps` RK3 steps each, the
 * state saved and restored around every trial), keeps the fastest column shape and
 * then the fastest row shape with it, drops captured step graphs, and remembers the
 * choice for later solvers of the same size, FFT precision and device.  Results
 * differ from the default shape by FP32 rounding only.  A tensor-core solver has one
 * row shape more, the last index: the row stage as split-precision DFT-GEMMs on the
 * tensor cores (its transforms then round like the column stage's). */
#define S2D_TUNE_MAX 8
typedef struct {
  int32_t phys_variants, spec_variants;   /* registered column / row shapes */
  int32_t phys_choice, spec_choice;       /* the shapes now in use */
  float phys_us[S2D_TUNE_MAX];            /* device time per RK3 step with each column shape */
  float spec_us[S2D_TUNE_MAX];            /* ... with each row shape (chosen column shape) */
} s2d_tune_report;
int s2d_autotune(s2d_solver* s, int steps, s2d_tune_report* report);
/* use registered shapes `phys` (column kernel) and `spec` (row kernel) from now on */
int s2d_tune_select(s2d_solver* s, int phys, int spec);
/* the name of registered shape `index` of the column (kind 0) or row (kind 1) kernel */
int s2d_tune_variant_name(s2d_solver* s, int kind, int index, char* out, int cap);

/* ---------------------------------------------------------------- headless image */
/* Renderer.render(encoder, solver, cfg) (render.js:63-87, render.wgsl:81-103) into a
 * host buffer of height*width RGBA8 pixels, row 0 at the top, instead of a canvas:
 * mode 0 dye, 1 vorticity, 2 dye over vorticity, 3 speed (render.js:4).  The
 * vorticity is the current state's (the reference shows the last stage's). */
#define S2D_RENDER_DYE 0
#define S2D_RENDER_VORTICITY 1
#define S2D_RENDER_DYE_OVER_VORTICITY 2
#define S2D_RENDER_SPEED 3
int s2d_render(s2d_solver* s, int mode, float exposure, float vort_scale, float dye_gain, int width, int height,
               void* rgba_out);

/* ---------------------------------------------------------------- step */
int s2d_encode_prime(s2d_solver* s);                                     /* solver.js:475-486 */
int s2d_encode_step(s2d_solver* s);                                      /* solver.js:488-521 */
int s2d_encode_dye(s2d_solver* s);                                       /* solver.js:523-536 */
/* encodeDye as the reference's three separate dispatches (advect_fwd, advect_back,
 * advect_corr, dye.wgsl:58-113); same result bits as s2d_encode_dye. */
int s2d_encode_dye_passes(s2d_solver* s);
int s2d_encode_reduce(s2d_solver* s);                                    /* solver.js:538-545 */
/* `substeps` repetitions of encodeStep (+ encodeDye, + encodeReduce per flags),
 * priming first when needed: the body of main.js:409-419. */
int s2d_step(s2d_solver* s, int substeps, unsigned flags);
/* As s2d_step, replayed from a captured CUDA graph of one substep. */
int s2d_step_graph(s2d_solver* s, int substeps, unsigned flags);

/* ---------------------------------------------------------------- diagnostics */
/* Diagnostics of the current state (solver.js:547-558): the zonal mean on the solver's
 * stream; the FP64 and fixed-point spectra on the solver's diagnostics stream, behind
 * the work enqueued so far, so that they run alongside the next step.  The library
 * orders its later calls after them where they would change what the spectra read (a
 * step call waits for them unless it is one fused step right after them), so the
 * results are those of the state at this call. */
int s2d_encode_diagnostics(s2d_solver* s);
/* solver.js:560-568: on the diagnostics stream, behind the spectra and the work enqueued
 * so far, copies the block the last s2d_encode_diagnostics filled and the [dt, speed]
 * slot current now. */
int s2d_copy_diagnostics(s2d_solver* s);
/* 1 when the copied diagnostics have landed in host memory, 0 otherwise. */
int s2d_poll_diagnostics(s2d_solver* s);
/* readDiagnostics() (solver.js:570-608): waits for the copy; S2D_NO_DATA when
 * nothing was copied (the JS null).  Spectrum, energy and enstrophy are FP64
 * reductions of the current state; zonal is the mean over x of u of the
 * velocity of the last RK stage-2 evaluation (the reference's packA.y). */
int s2d_read_diagnostics(s2d_solver* s, double* spectrum /* N/2+1 */, float* zonal /* N */,
                         double* energy, double* enstrophy, float* dt, float* max_speed);
/* The reference's fixed-point decoding of the same quantities
 * (spectrum.wgsl:19-39 accumulation, solver.js:591-602 decoding). */
int s2d_read_diagnostics_fixed(s2d_solver* s, float* spectrum /* N/2+1 */, float* energy,
                               float* enstrophy);

/* ---------------------------------------------------------------- stage hooks */
int s2d_get_buffer(s2d_solver* s, int id, void* host, size_t bytes);
int s2d_set_buffer(s2d_solver* s, int id, const void* host, size_t bytes);
/* Fft2D.forward/inverse(pass, name) (fft.js:81-101) on packA/packB/physZ/force;
 * other ids give S2D_ERR_UNREGISTERED.  Inverse scales 1/N per axis. */
int s2d_fft2(s2d_solver* s, int id, int inverse);
/* velocity_pack from state[state_index] into packA/packB (solver.wgsl:21-40). */
int s2d_velocity_pack(s2d_solver* s, int state_index);
/* nl_pack: packA/packB -> physZ, vel (solver.wgsl:42-54). */
int s2d_nl_pack(s2d_solver* s);
/* assemble: physZ, force, dt -> rhs (solver.wgsl:56-95). */
int s2d_assemble(s2d_solver* s);
/* rk3 stage update with the current phase's state ring (solver.wgsl:103-122). */
int s2d_rk3_stage(s2d_solver* s, int stage);
/* currentDye (solver.js:610-612): copies M*M*4 binary16 values. */
int s2d_get_dye(s2d_solver* s, uint16_t* out);
int s2d_set_dye(s2d_solver* s, const uint16_t* in);

/* ---------------------------------------------------------------- instrumentation */
/* Kernel classes timed by the profiler: the two fused stage kernels, the dye
 * passes, the pointer force (field + FFT) and everything else. */
#define S2D_PROF_PHYS_COLS 0
#define S2D_PROF_SPEC_ROWS 1
#define S2D_PROF_DYE 2
#define S2D_PROF_FORCE 3
#define S2D_PROF_OTHER 4
#define S2D_PROF_CLASSES 5
/* enable != 0 starts recording a CUDA event pair around every kernel class the
 * step entry points launch (no reference counterpart); 0 stops.  With
 * s2d_step_graph the events are nodes of the captured graph and each replay is
 * synchronized and read, so the times are device times without host gaps. */
int s2d_profile(s2d_solver* s, int enable);
/* Synchronizes, then returns the summed device time (ms) and launch count per
 * class since the last read, and clears them. */
int s2d_profile_read(s2d_solver* s, double* ms /* S2D_PROF_CLASSES */, int* launches /* S2D_PROF_CLASSES */);

/* ---------------------------------------------------------------- allocation-free CFL step */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- applications that reserve all GPU memory up front for their own
 * allocator, or whose frame loop may not call cudaMalloc/cudaFree because those
 * calls can synchronize the device -- this computes what s2d_encode_reduce
 * computes, [dt, max |u|+|v|] with dt = clamp(cfl * (2 pi/n) / max, dt_min,
 * dt_max) (dt_max when the maximum is <= 1e-8), from a caller-owned device
 * velocity field `vel` (n*n interleaved (u, v) floats) into the caller-owned
 * device buffer `dt_out` (2 floats), enqueued on `stream` (a cudaStream_t;
 * NULL is the default stream), and allocates nothing.  Its only scratch is a
 * static device array of S2D_CFL_STATIC_MAX_PARTIALS floats (16 KiB) that every
 * GPU loading the library holds until the process exits, so n is limited to
 * S2D_CFL_STATIC_MAX_N; larger n is rejected with S2D_ERR_ARG.  The first call
 * in each CUDA context (a device's primary context, or a context the caller made
 * current) looks up that array's device address there (cudaGetSymbolAddress);
 * make that first call before any stream capture.  All
 * calls on a device share the array: calls that overlap on the GPU (other
 * streams, other host threads) race and must be ordered by the caller. */
#define S2D_CFL_STATIC_MAX_N 4096
#define S2D_CFL_STATIC_MAX_PARTIALS 4096
int s2d_cfl_dt_static(const void* vel, int n, float cfl, float dt_min, float dt_max, void* dt_out, void* stream);

/* ---------------------------------------------------------------- ensemble */
/* Many independent instances of uneven sizes stepped together, each with its own
 * viscosity, beta, drag and forcing (no reference counterpart beyond running
 * many Solvers). */
typedef struct s2d_instance_desc {
  int32_t n;              /* 64..1024, power of two */
  float beta, drag, nu_h; /* nu_h directly (not the rate) */
  int32_t hyper_p;
  float dt;               /* fixed step of this instance */
  float force_amp, force_k, force_width;
  uint32_t seed;
} s2d_instance_desc;

typedef struct s2d_ensemble s2d_ensemble;

int s2d_ensemble_create(const s2d_instance_desc* descs, int count, int device,
                        s2d_ensemble** out);
int s2d_ensemble_destroy(s2d_ensemble* e);
int s2d_ensemble_get_stream(s2d_ensemble* e, void** stream);
int s2d_ensemble_synchronize(s2d_ensemble* e);
/* Band-limited complex Gaussian initial spectra (kmin <= |k| <= kmax, rms
 * vorticity `rms`) for every instance, seeded by the descriptor seeds. */
int s2d_ensemble_seed_band(s2d_ensemble* e, float kmin, float kmax, float rms);
int s2d_ensemble_set_state(s2d_ensemble* e, int index, const float* spectrum /* n*n*2 */);
int s2d_ensemble_get_state(s2d_ensemble* e, int index, float* spectrum /* n*n*2 */);
/* `steps` RK3 steps of every instance; use_graph replays a captured step. */
int s2d_ensemble_step(s2d_ensemble* e, int steps, int use_graph);
/* FP64 energy and enstrophy of every instance (arrays of `count`). */
int s2d_ensemble_energy(s2d_ensemble* e, double* energy, double* enstrophy);
/* The autotuner for an ensemble (no reference counterpart): times the registered
 * resident-CTA shapes of the persistent column and row kernels over `steps` RK3 steps
 * of this ensemble (its state saved and restored bit for bit), keeps the fastest, and
 * drops captured step graphs.  The shapes differ in register allocation only. */
int s2d_ensemble_autotune(s2d_ensemble* e, int steps, s2d_tune_report* report);
int s2d_ensemble_tune_variant_name(s2d_ensemble* e, int kind, int index, char* out, int cap);
/* Pin the column / row launch shapes (indices as in the report above; drops captured
 * step graphs).  No reference counterpart. */
int s2d_ensemble_tune_select(s2d_ensemble* e, int phys, int spec);

#ifdef __cplusplus
}
#endif
#endif /* S2D_H */
