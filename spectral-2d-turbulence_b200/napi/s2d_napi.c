/* s2d_napi.c -- Node-API addon over the C ABI of libs2d.so (include/s2d.h).
 *
 * The reference drives its solver from JavaScript (src/gpu/solver.js, class Solver,
 * lines 49-630; src/gpu/fft.js; src/gpu/device.js).  This addon is the thin native
 * layer a Node host loads in place of the WebGPU device: one external handle per
 * solver, one exported function per C entry point.  The JavaScript class with the
 * reference's method names is solver_b200.js next to this file.
 *
 * Conventions
 *  - every function takes the handle first; a negative status becomes a thrown JS Error
 *    whose message is s2d_last_error() and whose `code` is the status (the reference
 *    throws Error objects, fft.js:28,84; shaders.js:50-53; device.js:10-16);
 *  - typed arrays are passed by pointer, never copied on the JS side;
 *  - readDiagnostics returns a Promise (solver.js:570-608 is async): the copy's CUDA
 *    event is waited for on a libuv worker thread by polling s2d_poll_diagnostics, and
 *    the read itself (s2d_read_diagnostics) runs on the JS thread in the completion
 *    callback, so no other entry point ever runs concurrently with it.  The Promise
 *    resolves to null when nothing was copied, as the reference's does.
 * Node-API version 8 (Node >= 12.22) is enough.
 */
#define NAPI_VERSION 8
#include <node_api.h>

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "s2d.h"

/* ------------------------------------------------------------------ handle */
typedef struct {
  s2d_solver* s;
  int32_t n, m, nbins;
  int pending;   /* a diagnostics copy is in flight (solver.js readState 1) */
  int reading;   /* a readDiagnostics Promise is outstanding */
} js_solver;

static void finalize_solver(napi_env env, void* data, void* hint) {
  (void)env;
  (void)hint;
  js_solver* h = (js_solver*)data;
  if (h->s) s2d_destroy(h->s);
  free(h);
}

static napi_value throw_status(napi_env env, int st) {
  char code[16];
  snprintf(code, sizeof code, "%d", st);
  const char* msg = s2d_last_error();
  napi_throw_error(env, code, msg && msg[0] ? msg : s2d_status_string(st));
  return NULL;
}
#define CALL(expr)                              \
  do {                                          \
    const int st_ = (expr);                     \
    if (st_ < 0) return throw_status(env, st_); \
  } while (0)
#define NAPI(expr)                                                  \
  do {                                                              \
    if ((expr) != napi_ok) {                                        \
      napi_throw_error(env, NULL, "Node-API call failed: " #expr); \
      return NULL;                                                  \
    }                                                               \
  } while (0)

static napi_value undefined(napi_env env) {
  napi_value u;
  napi_get_undefined(env, &u);
  return u;
}

/* the first `want` arguments (missing ones read as undefined) */
static int args(napi_env env, napi_callback_info info, size_t want, napi_value* argv) {
  size_t argc = want;
  if (napi_get_cb_info(env, info, &argc, argv, NULL, NULL) != napi_ok) return 0;
  for (size_t i = argc; i < want; ++i) napi_get_undefined(env, &argv[i]);
  return 1;
}

static js_solver* handle_of(napi_env env, napi_value v) {
  void* p = NULL;
  if (napi_get_value_external(env, v, &p) != napi_ok || !p) {
    napi_throw_type_error(env, NULL, "expected a solver handle");
    return NULL;
  }
  js_solver* h = (js_solver*)p;
  if (!h->s) {
    napi_throw_error(env, "-4", "solver destroyed");   /* S2D_ERR_DESTROYED, solver.js:571,614-615 */
    return NULL;
  }
  return h;
}
#define HANDLE(v)                        \
  js_solver* h = handle_of(env, (v));    \
  if (!h) return NULL

static double num_or(napi_env env, napi_value v, double dflt) {
  napi_valuetype t;
  double d = dflt;
  if (napi_typeof(env, v, &t) == napi_ok && t == napi_number) napi_get_value_double(env, v, &d);
  return d;
}
static double prop(napi_env env, napi_value obj, const char* key, double dflt) {
  bool has = false;
  napi_value v;
  if (napi_has_named_property(env, obj, key, &has) != napi_ok || !has) return dflt;
  if (napi_get_named_property(env, obj, key, &v) != napi_ok) return dflt;
  return num_or(env, v, dflt);
}
static napi_value make_num(napi_env env, double d) {
  napi_value v;
  napi_create_double(env, d, &v);
  return v;
}
static void set_num(napi_env env, napi_value obj, const char* key, double d) {
  napi_set_named_property(env, obj, key, make_num(env, d));
}

/* typed array argument: element pointer and count, checked against the wanted type */
static void* typed(napi_env env, napi_value v, napi_typedarray_type want, size_t* count) {
  bool is = false;
  if (napi_is_typedarray(env, v, &is) != napi_ok || !is) {
    napi_throw_type_error(env, NULL, "expected a typed array");
    return NULL;
  }
  napi_typedarray_type t;
  size_t len = 0, off = 0;
  void* data = NULL;
  napi_value ab;
  if (napi_get_typedarray_info(env, v, &t, &len, &data, &ab, &off) != napi_ok || t != want) {
    napi_throw_type_error(env, NULL, "typed array of the wrong element type");
    return NULL;
  }
  *count = len;
  return data;
}

static napi_value new_typed(napi_env env, napi_typedarray_type t, size_t count, size_t elem, void** data) {
  napi_value ab, arr;
  if (napi_create_arraybuffer(env, count * elem, data, &ab) != napi_ok) return NULL;
  if (napi_create_typedarray(env, t, count, ab, 0, &arr) != napi_ok) return NULL;
  return arr;
}

/* ------------------------------------------------------------------ library-level */
/* radixSchedule(n) -> {stages, hasRadix2} (fft.js:20-31) */
static napi_value js_radix_schedule(napi_env env, napi_callback_info info) {
  napi_value a[1];
  if (!args(env, info, 1, a)) return NULL;
  int32_t n = 0, stages = 0, r2 = 0;
  NAPI(napi_get_value_int32(env, a[0], &n));
  CALL(s2d_radix_schedule(n, &stages, &r2));
  napi_value o;
  NAPI(napi_create_object(env, &o));
  set_num(env, o, "stages", stages);
  napi_value b;
  napi_get_boolean(env, r2 != 0, &b);
  napi_set_named_property(env, o, "hasRadix2", b);
  return o;
}

/* supportedGrids() -> number[] (device.js:44-52) */
static napi_value js_supported_grids(napi_env env, napi_callback_info info) {
  (void)info;
  int32_t grids[16];
  int32_t count = 0;
  CALL(s2d_supported_grids(grids, 16, &count));
  napi_value arr;
  NAPI(napi_create_array_with_length(env, (size_t)count, &arr));
  for (int32_t i = 0; i < count; ++i) napi_set_element(env, arr, (uint32_t)i, make_num(env, grids[i]));
  return arr;
}

/* ------------------------------------------------------------------ lifecycle */
/* create(n, dyeScale, fftPrecision, device) -> handle (solver.js:71-75) */
static napi_value js_create(napi_env env, napi_callback_info info) {
  napi_value a[4];
  if (!args(env, info, 4, a)) return NULL;
  const int32_t n = (int32_t)num_or(env, a[0], 256), scale = (int32_t)num_or(env, a[1], 2);
  const int32_t fft = (int32_t)num_or(env, a[2], S2D_FFT_FP32), dev = (int32_t)num_or(env, a[3], 0);
  s2d_solver* s = NULL;
  CALL(s2d_create(n, scale, fft, dev, &s));
  js_solver* h = (js_solver*)calloc(1, sizeof(js_solver));
  if (!h) {
    s2d_destroy(s);
    napi_throw_error(env, NULL, "out of host memory");
    return NULL;
  }
  h->s = s;
  s2d_info inf;
  if (s2d_get_info(s, &inf) == S2D_OK) {
    h->n = inf.n;
    h->m = inf.m;
    h->nbins = inf.nbins;
  }
  napi_value out;
  if (napi_create_external(env, h, finalize_solver, NULL, &out) != napi_ok) {
    finalize_solver(env, h, NULL);
    napi_throw_error(env, NULL, "napi_create_external failed");
    return NULL;
  }
  return out;
}

/* destroy(h) (solver.js:614-629): frees the solver now; later calls throw */
static napi_value js_destroy(napi_env env, napi_callback_info info) {
  napi_value a[1];
  if (!args(env, info, 1, a)) return NULL;
  void* p = NULL;
  if (napi_get_value_external(env, a[0], &p) == napi_ok && p) {
    js_solver* h = (js_solver*)p;
    if (h->s && !h->reading) {
      s2d_destroy(h->s);
      h->s = NULL;
    } else if (h->s) {
      /* a diagnostics read is in flight: its completion callback frees the solver */
      h->reading = 2;
    }
  }
  return undefined(env);
}

/* info(h) -> {n, m, nbins, phase, dyeParity, stepIndex, primed, fftPrecision, nuH, simTime} */
static napi_value js_info(napi_env env, napi_callback_info info) {
  napi_value a[1];
  if (!args(env, info, 1, a)) return NULL;
  HANDLE(a[0]);
  s2d_info inf;
  CALL(s2d_get_info(h->s, &inf));
  napi_value o;
  NAPI(napi_create_object(env, &o));
  set_num(env, o, "n", inf.n);
  set_num(env, o, "m", inf.m);
  set_num(env, o, "nbins", inf.nbins);
  set_num(env, o, "phase", inf.phase);
  set_num(env, o, "dyeParity", inf.dye_parity);
  set_num(env, o, "stepIndex", inf.step_index);
  set_num(env, o, "primed", inf.primed);
  set_num(env, o, "fftPrecision", inf.fft_precision);
  set_num(env, o, "nuH", inf.nu_h);
  set_num(env, o, "simTime", inf.sim_time);
  return o;
}

/* setSimTime(h, t) -- the host advances simTime from the diagnostics dt (main.js:441-443) */
static napi_value js_set_sim_time(napi_env env, napi_callback_info info) {
  napi_value a[2];
  if (!args(env, info, 2, a)) return NULL;
  HANDLE(a[0]);
  CALL(s2d_set_sim_time(h->s, num_or(env, a[1], 0.0)));
  return undefined(env);
}

/* ------------------------------------------------------------------ parameters */
/* configure(h, cfg) (solver.js:306-324): the main.js config keys */
static napi_value js_configure(napi_env env, napi_callback_info info) {
  napi_value a[2];
  if (!args(env, info, 2, a)) return NULL;
  HANDLE(a[0]);
  s2d_params p;
  p.beta = (float)prop(env, a[1], "beta", 0.0);
  p.drag = (float)prop(env, a[1], "drag", 0.0);
  p.viscosity = (float)prop(env, a[1], "viscosity", 0.0);
  p.hyper_p = (int32_t)prop(env, a[1], "hyperP", 4);
  p.force_amp = (float)prop(env, a[1], "forceAmp", 0.0);
  p.force_k = (float)prop(env, a[1], "forceK", 20.0);
  p.force_width = (float)prop(env, a[1], "forceWidth", 2.0);
  p.cfl = (float)prop(env, a[1], "cfl", 0.5);
  p.dt_min = (float)prop(env, a[1], "dtMin", 1e-5);
  p.dt_max = (float)prop(env, a[1], "dtMax", 0.05);
  p.dye_fade = (float)prop(env, a[1], "dyeFade", 1.0);
  CALL(s2d_configure(h->s, &p));
  return undefined(env);
}

/* setSplats(h, list) (solver.js:326-345): at most MAX_SPLATS of {x, y, dx, dy, color[3],
 * radius, amp, dyeAmp}, as built by ui/pointer.js */
static napi_value js_set_splats(napi_env env, napi_callback_info info) {
  napi_value a[2];
  if (!args(env, info, 2, a)) return NULL;
  HANDLE(a[0]);
  s2d_splat list[S2D_MAX_SPLATS];
  uint32_t len = 0;
  bool is_arr = false;
  if (napi_is_array(env, a[1], &is_arr) == napi_ok && is_arr) napi_get_array_length(env, a[1], &len);
  if (len > S2D_MAX_SPLATS) len = S2D_MAX_SPLATS;   /* Math.min(list.length, MAX_SPLATS) */
  for (uint32_t i = 0; i < len; ++i) {
    napi_value e, col;
    NAPI(napi_get_element(env, a[1], i, &e));
    s2d_splat* s = &list[i];
    s->x = (float)prop(env, e, "x", 0.0);
    s->y = (float)prop(env, e, "y", 0.0);
    s->dx = (float)prop(env, e, "dx", 0.0);
    s->dy = (float)prop(env, e, "dy", 0.0);
    s->radius = (float)prop(env, e, "radius", 0.0);
    s->amp = (float)prop(env, e, "amp", 0.0);
    s->dye_amp = (float)prop(env, e, "dyeAmp", 0.0);
    s->color[0] = s->color[1] = s->color[2] = 0.f;
    bool has = false;
    if (napi_has_named_property(env, e, "color", &has) == napi_ok && has &&
        napi_get_named_property(env, e, "color", &col) == napi_ok) {
      for (uint32_t c = 0; c < 3; ++c) {
        napi_value cv;
        if (napi_get_element(env, col, c, &cv) == napi_ok) s->color[c] = (float)num_or(env, cv, 0.0);
      }
    }
  }
  CALL(s2d_set_splats(h->s, list, (int)len));
  return undefined(env);
}

/* ------------------------------------------------------------------ seeding */
/* seed(h, k0, amplitude, seed) (solver.js:347-359) */
static napi_value js_seed(napi_env env, napi_callback_info info) {
  napi_value a[4];
  if (!args(env, info, 4, a)) return NULL;
  HANDLE(a[0]);
  CALL(s2d_seed(h->s, num_or(env, a[1], 14.0), num_or(env, a[2], 6.0), (uint32_t)num_or(env, a[3], 1.0)));
  return undefined(env);
}

/* seedPhysical(h, Float32Array N*N) (solver.js:361-382) */
static napi_value js_seed_physical(napi_env env, napi_callback_info info) {
  napi_value a[2];
  if (!args(env, info, 2, a)) return NULL;
  HANDLE(a[0]);
  size_t count = 0;
  const float* f = (const float*)typed(env, a[1], napi_float32_array, &count);
  if (!f) return NULL;
  if (count != (size_t)h->n * (size_t)h->n) {
    napi_throw_range_error(env, NULL, "seedPhysical expects n*n values");
    return NULL;
  }
  CALL(s2d_seed_physical(h->s, f));
  return undefined(env);
}

/* reset(h, field | null, k0, amplitude, seed, dyePattern) (solver.js:420-444) */
static napi_value js_reset(napi_env env, napi_callback_info info) {
  napi_value a[6];
  if (!args(env, info, 6, a)) return NULL;
  HANDLE(a[0]);
  const float* field = NULL;
  napi_valuetype t;
  napi_typeof(env, a[1], &t);
  if (t != napi_null && t != napi_undefined) {
    size_t count = 0;
    field = (const float*)typed(env, a[1], napi_float32_array, &count);
    if (!field) return NULL;
    if (count != (size_t)h->n * (size_t)h->n) {
      napi_throw_range_error(env, NULL, "reset field expects n*n values");
      return NULL;
    }
  }
  CALL(s2d_reset(h->s, field, num_or(env, a[2], 14.0), num_or(env, a[3], 6.0), (uint32_t)num_or(env, a[4], 1.0),
                 (int)num_or(env, a[5], S2D_DYE_BANDS)));
  h->pending = 0;
  return undefined(env);
}

/* paintDye(h, pattern) (solver.js:446-473): S2D_DYE_NONE / S2D_DYE_BANDS */
static napi_value js_paint_dye(napi_env env, napi_callback_info info) {
  napi_value a[2];
  if (!args(env, info, 2, a)) return NULL;
  HANDLE(a[0]);
  CALL(s2d_paint_dye(h->s, (int)num_or(env, a[1], S2D_DYE_BANDS)));
  return undefined(env);
}

/* ------------------------------------------------------------------ stepping */
#define SIMPLE(jsname, fn)                                          \
  static napi_value jsname(napi_env env, napi_callback_info info) { \
    napi_value a[1];                                                \
    if (!args(env, info, 1, a)) return NULL;                        \
    HANDLE(a[0]);                                                   \
    CALL(fn(h->s));                                                 \
    return undefined(env);                                          \
  }
SIMPLE(js_encode_prime, s2d_encode_prime)             /* solver.js:475-486 */
SIMPLE(js_encode_step, s2d_encode_step)               /* solver.js:488-521 */
SIMPLE(js_encode_dye, s2d_encode_dye)                 /* solver.js:523-536 */
SIMPLE(js_encode_reduce, s2d_encode_reduce)           /* solver.js:538-545 */
SIMPLE(js_encode_diagnostics, s2d_encode_diagnostics) /* solver.js:547-558 */
SIMPLE(js_synchronize, s2d_synchronize)

/* copyDiagnostics(h) (solver.js:560-568): ignored while a copy is in flight */
static napi_value js_copy_diagnostics(napi_env env, napi_callback_info info) {
  napi_value a[1];
  if (!args(env, info, 1, a)) return NULL;
  HANDLE(a[0]);
  if (h->pending) return undefined(env);
  CALL(s2d_copy_diagnostics(h->s));
  h->pending = 1;
  return undefined(env);
}

/* step(h, substeps, flags, graph): substeps of the main.js:413-419 loop in one call */
static napi_value js_step(napi_env env, napi_callback_info info) {
  napi_value a[4];
  if (!args(env, info, 4, a)) return NULL;
  HANDLE(a[0]);
  const int substeps = (int)num_or(env, a[1], 1.0);
  const unsigned flags = (unsigned)num_or(env, a[2], S2D_STEP_DYE | S2D_STEP_REDUCE);
  bool graph = false;
  napi_get_value_bool(env, a[3], &graph);
  if (graph) CALL(s2d_step_graph(h->s, substeps, flags));
  else CALL(s2d_step(h->s, substeps, flags));
  return undefined(env);
}

/* ------------------------------------------------------------------ diagnostics (async) */
typedef struct {
  js_solver* h;
  napi_deferred deferred;
  napi_async_work work;
  int ready;   /* the copy's event completed within the limit */
} read_job;

/* worker thread: wait (polling, at most 10 s) for the copy's event */
static void read_execute(napi_env env, void* data) {
  (void)env;
  read_job* j = (read_job*)data;
  const struct timespec nap = {0, 100000};   /* 100 us */
  for (int i = 0; i < 100000; ++i) {
    if (s2d_poll_diagnostics(j->h->s) == 1) {
      j->ready = 1;
      return;
    }
    nanosleep(&nap, NULL);
  }
}

/* JS thread: read the pinned block and resolve with the reference's result shape */
static void read_complete(napi_env env, napi_status status, void* data) {
  read_job* j = (read_job*)data;
  js_solver* h = j->h;
  napi_value result = NULL;
  if (status == napi_ok && j->ready && h->s) {
    const int nb = h->nbins, n = h->n;
    double* spec = (double*)malloc(sizeof(double) * (size_t)nb);
    float* zonal = NULL;
    napi_value zarr = new_typed(env, napi_float32_array, (size_t)n, sizeof(float), (void**)&zonal);
    double e = 0, z = 0;
    float dt = 0, sp = 0;
    const int st = spec && zarr ? s2d_read_diagnostics(h->s, spec, zonal, &e, &z, &dt, &sp) : S2D_ERR_ARG;
    if (st == S2D_OK) {
      /* spectrum as Float32Array(N/2+1), like the reference's decoded bins (solver.js:591-599) */
      float* s32 = NULL;
      napi_value sarr = new_typed(env, napi_float32_array, (size_t)nb, sizeof(float), (void**)&s32);
      if (sarr) {
        for (int i = 0; i < nb; ++i) s32[i] = (float)spec[i];
        napi_create_object(env, &result);
        napi_set_named_property(env, result, "spectrum", sarr);
        napi_set_named_property(env, result, "zonal", zarr);
        set_num(env, result, "energy", e);
        set_num(env, result, "enstrophy", z);
        set_num(env, result, "dt", dt);
        set_num(env, result, "maxSpeed", sp);
      }
    }
    free(spec);
  }
  h->pending = 0;
  if (!result) napi_get_null(env, &result);   /* solver.js:603-604 resolves null on failure */
  napi_resolve_deferred(env, j->deferred, result);
  napi_delete_async_work(env, j->work);
  if (h->reading == 2 && h->s) {   /* destroy() was called while the read was in flight */
    s2d_destroy(h->s);
    h->s = NULL;
  }
  h->reading = 0;
  free(j);
}

/* readDiagnostics(h) -> Promise<{spectrum, zonal, energy, enstrophy, dt, maxSpeed} | null> */
static napi_value js_read_diagnostics(napi_env env, napi_callback_info info) {
  napi_value a[1];
  if (!args(env, info, 1, a)) return NULL;
  napi_value promise;
  napi_deferred deferred;
  NAPI(napi_create_promise(env, &deferred, &promise));
  void* p = NULL;
  js_solver* h = NULL;
  if (napi_get_value_external(env, a[0], &p) == napi_ok) h = (js_solver*)p;
  if (!h || !h->s || !h->pending || h->reading) {
    /* destroyed, nothing copied, or a read already outstanding (solver.js:571-573) */
    napi_value nul;
    napi_get_null(env, &nul);
    napi_resolve_deferred(env, deferred, nul);
    return promise;
  }
  read_job* j = (read_job*)calloc(1, sizeof(read_job));
  if (!j) {
    napi_value nul;
    napi_get_null(env, &nul);
    napi_resolve_deferred(env, deferred, nul);
    return promise;
  }
  j->h = h;
  j->deferred = deferred;
  napi_value name;
  NAPI(napi_create_string_utf8(env, "s2d.readDiagnostics", NAPI_AUTO_LENGTH, &name));
  NAPI(napi_create_async_work(env, NULL, name, read_execute, read_complete, j, &j->work));
  h->reading = 1;
  NAPI(napi_queue_async_work(env, j->work));
  return promise;
}

/* ------------------------------------------------------------------ buffers */
/* currentDye(h) -> Uint16Array(M*M*4) of binary16 rgba (the texture getter, solver.js:610-612) */
static napi_value js_current_dye(napi_env env, napi_callback_info info) {
  napi_value a[1];
  if (!args(env, info, 1, a)) return NULL;
  HANDLE(a[0]);
  uint16_t* data = NULL;
  napi_value arr = new_typed(env, napi_uint16_array, (size_t)h->m * (size_t)h->m * 4, sizeof(uint16_t), (void**)&data);
  if (!arr) return NULL;
  CALL(s2d_get_dye(h->s, data));
  return arr;
}

/* getBuffer(h, id) -> Float32Array; setBuffer(h, id, Float32Array): the per-stage test hooks
 * of tests/index.html (packA, packB, physZ, rhs, force, state[i], vel, dt) */
static size_t buffer_floats(const js_solver* h, int id) {
  if (id == S2D_BUF_DT) return 4;
  return (size_t)h->n * (size_t)h->n * 2;
}
static napi_value js_get_buffer(napi_env env, napi_callback_info info) {
  napi_value a[2];
  if (!args(env, info, 2, a)) return NULL;
  HANDLE(a[0]);
  const int id = (int)num_or(env, a[1], -1);
  const size_t count = buffer_floats(h, id);
  float* data = NULL;
  napi_value arr = new_typed(env, napi_float32_array, count, sizeof(float), (void**)&data);
  if (!arr) return NULL;
  CALL(s2d_get_buffer(h->s, id, data, count * sizeof(float)));
  return arr;
}
static napi_value js_set_buffer(napi_env env, napi_callback_info info) {
  napi_value a[3];
  if (!args(env, info, 3, a)) return NULL;
  HANDLE(a[0]);
  const int id = (int)num_or(env, a[1], -1);
  size_t count = 0;
  const float* data = (const float*)typed(env, a[2], napi_float32_array, &count);
  if (!data) return NULL;
  CALL(s2d_set_buffer(h->s, id, data, count * sizeof(float)));
  return undefined(env);
}

/* fft2(h, id, inverse) -- Fft2D.forward / inverse on a registered buffer (fft.js:81-101) */
static napi_value js_fft2(napi_env env, napi_callback_info info) {
  napi_value a[3];
  if (!args(env, info, 3, a)) return NULL;
  HANDLE(a[0]);
  bool inv = false;
  napi_get_value_bool(env, a[2], &inv);
  CALL(s2d_fft2(h->s, (int)num_or(env, a[1], -1), inv ? 1 : 0));
  return undefined(env);
}

/* ------------------------------------------------------------------ module */
static napi_value init(napi_env env, napi_value exports) {
  const napi_property_descriptor d[] = {
      {"radixSchedule", NULL, js_radix_schedule, NULL, NULL, NULL, napi_default, NULL},
      {"supportedGrids", NULL, js_supported_grids, NULL, NULL, NULL, napi_default, NULL},
      {"create", NULL, js_create, NULL, NULL, NULL, napi_default, NULL},
      {"destroy", NULL, js_destroy, NULL, NULL, NULL, napi_default, NULL},
      {"info", NULL, js_info, NULL, NULL, NULL, napi_default, NULL},
      {"setSimTime", NULL, js_set_sim_time, NULL, NULL, NULL, napi_default, NULL},
      {"configure", NULL, js_configure, NULL, NULL, NULL, napi_default, NULL},
      {"setSplats", NULL, js_set_splats, NULL, NULL, NULL, napi_default, NULL},
      {"seed", NULL, js_seed, NULL, NULL, NULL, napi_default, NULL},
      {"seedPhysical", NULL, js_seed_physical, NULL, NULL, NULL, napi_default, NULL},
      {"reset", NULL, js_reset, NULL, NULL, NULL, napi_default, NULL},
      {"paintDye", NULL, js_paint_dye, NULL, NULL, NULL, napi_default, NULL},
      {"encodePrime", NULL, js_encode_prime, NULL, NULL, NULL, napi_default, NULL},
      {"encodeStep", NULL, js_encode_step, NULL, NULL, NULL, napi_default, NULL},
      {"encodeDye", NULL, js_encode_dye, NULL, NULL, NULL, napi_default, NULL},
      {"encodeReduce", NULL, js_encode_reduce, NULL, NULL, NULL, napi_default, NULL},
      {"encodeDiagnostics", NULL, js_encode_diagnostics, NULL, NULL, NULL, napi_default, NULL},
      {"copyDiagnostics", NULL, js_copy_diagnostics, NULL, NULL, NULL, napi_default, NULL},
      {"readDiagnostics", NULL, js_read_diagnostics, NULL, NULL, NULL, napi_default, NULL},
      {"step", NULL, js_step, NULL, NULL, NULL, napi_default, NULL},
      {"synchronize", NULL, js_synchronize, NULL, NULL, NULL, napi_default, NULL},
      {"currentDye", NULL, js_current_dye, NULL, NULL, NULL, napi_default, NULL},
      {"getBuffer", NULL, js_get_buffer, NULL, NULL, NULL, napi_default, NULL},
      {"setBuffer", NULL, js_set_buffer, NULL, NULL, NULL, napi_default, NULL},
      {"fft2", NULL, js_fft2, NULL, NULL, NULL, napi_default, NULL},
  };
  if (napi_define_properties(env, exports, sizeof(d) / sizeof(d[0]), d) != napi_ok) return NULL;
  return exports;
}

NAPI_MODULE(NODE_GYP_MODULE_NAME, init)
