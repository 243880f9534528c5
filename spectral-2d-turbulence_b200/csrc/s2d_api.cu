// s2d_api.cu -- C ABI (include/s2d.h) over the sm_100a kernels.
//
// The solver object mirrors src/gpu/solver.js `class Solver`: it owns every
// device buffer (the triple-buffered state ring, the FFT work buffers, the dye
// textures as binary16 arrays) and one CUDA stream on which all of its work is
// ordered, the way the reference encodes everything into one compute pass.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/s2d.h"
#include "s2d_aux_kernels.cuh"
#include "s2d_ops.cuh"
#include "s2d_tc.cuh"
#include "s2d_tc_cols.cuh"
#include "s2d_tc_lines.h"
#include "s2d_render.cuh"

using namespace s2d;

static thread_local std::string g_last_error;

static int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

namespace s2d {
// error text of the ensemble translation unit, reported by s2d_last_error()
const char* ens_set_error(const std::string& m) {
  g_last_error = m;
  return g_last_error.c_str();
}
}  // namespace s2d
#define S2D_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(S2D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
  } while (0)
#define S2D_LAUNCHED()                                                                       \
  do {                                                                                       \
    cudaError_t e_ = cudaGetLastError();                                                     \
    if (e_ != cudaSuccess)                                                                   \
      return fail(S2D_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_));    \
  } while (0)

// ------------------------------------------------------------------ size dispatch
namespace s2d {
const NOps* ops_n32();
const NOps* ops_n64();
const NOps* ops_n128();
const NOps* ops_n256();
const NOps* ops_n512();
const NOps* ops_n1024();
const NOps* ops_n2048();
const NOps* ops_n4096();
}  // namespace s2d

static const NOps* ops_for(int n) {
  switch (n) {
    case 32: return ops_n32();
    case 64: return ops_n64();
    case 128: return ops_n128();
    case 256: return ops_n256();
    case 512: return ops_n512();
    case 1024: return ops_n1024();
    case 2048: return ops_n2048();
    case 4096: return ops_n4096();
    default: return nullptr;
  }
}

static bool radix_ok(int n, int* stages, int* has_r2) {
  if (n < 2) return false;
  int s = 0, m = n;
  while (m % 4 == 0) {
    ++s;
    m /= 4;
  }
  if (m != 1 && m != 2) return false;
  if (stages) *stages = s;
  if (has_r2) *has_r2 = (m == 2);
  return true;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
    else prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

static int check_device(int dev) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return fail(S2D_ERR_NO_DEVICE, "no CUDA device available");
  if (dev < 0 || dev >= count) return fail(S2D_ERR_ARG, "device index out of range");
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return fail(S2D_ERR_NO_DEVICE, "device query failed");
  if (p.major != 10) return fail(S2D_ERR_NO_DEVICE, "this library is built for sm_100a (B200) only");
  return S2D_OK;
}

// ------------------------------------------------------------------ solver object
struct GraphKey {
  int phase, slot, parity;
  unsigned flags;
  int ptr, prof;
  bool operator<(const GraphKey& o) const {
    return std::tie(phase, slot, parity, flags, ptr, prof) <
           std::tie(o.phase, o.slot, o.parity, o.flags, o.ptr, o.prof);
  }
};

// a captured substep; when profiling, it carries event-record nodes around its kernels
struct GraphEntry {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> events;
};

// One diagnostics block: FP64 bins + energy + enstrophy [nbins + 2], u32 fixed-point bins
// + totals [nbins + 2], zonal mean [n].
static size_t diag_block_bytes(int nbins, int n) {
  return (sizeof(double) + sizeof(uint32_t)) * (size_t)(nbins + 2) + sizeof(float) * (size_t)n;
}
// Two blocks, used in turn, then the two dt slots: [block 0][block 1][dt slots], each part
// 16-byte aligned.  Each diagnostics call fills one block and clears the sums of the other
// for the next call (no separate clear).
static size_t diag_block_stride(int nbins, int n) { return (diag_block_bytes(nbins, n) + 15) & ~size_t(15); }
static size_t diag_block_offset(int nbins, int n, int b) { return (size_t)b * diag_block_stride(nbins, n); }
static size_t diag_dt_offset(int nbins, int n) { return 2 * diag_block_stride(nbins, n); }
static size_t diag_alloc_bytes(int nbins, int n) { return diag_dt_offset(nbins, n) + 4 * sizeof(float); }

constexpr int kUploadSlots = 8;
constexpr size_t kUploadSlotBytes = 512;
// the parameter and splat blocks sit back to back in one device allocation, so that a
// configure() and a setSplats() before a step travel in one copy
constexpr size_t kConstBytes = sizeof(DevParams) + sizeof(DevSplats);
static_assert(kConstBytes <= kUploadSlotBytes, "upload slot");
static_assert(sizeof(DevParams) % 16 == 0, "splat block alignment");

struct s2d_solver {
  int dev = 0, n = 0, m = 0, nbins = 0, dye_scale = 1, fft_precision = 0;
  cudaStream_t stream = nullptr;        // every launch except the diagnostics below (high priority)
  // Diagnostics stream (low priority): the k-space spectra of encodeDiagnostics and the
  // readback copies run there, behind the work the main stream had enqueued, and alongside
  // the next step.  The spectra read state[phase] of the step before them, which the next
  // fused step reads but does not write; every other call that enqueues device work first
  // orders the main stream after them (diag_order).
  cudaStream_t diag_stream = nullptr;
  cudaEvent_t diag_ready = nullptr;     // main-stream point the diagnostics stream waits for
  cudaEvent_t diag_done = nullptr;      // the last spectra launch has finished
  bool diag_outstanding = false;        // diag_done not yet waited for by the main stream
  int diag_age = 0;                     // steps enqueued since the outstanding spectra launch
  int in_step = 0;                      // inside a step call (its inner entry points do not order)
  const NOps* ops = nullptr;
  float2* state[3] = {nullptr, nullptr, nullptr};
  float2 *packA = nullptr, *packB = nullptr, *physZ = nullptr, *rhs = nullptr, *force = nullptr,
         *vel = nullptr, *tw = nullptr;
  float* dtbuf = nullptr;      // 2 slots x [dt, speed], at the end of diag's allocation
  float* partials = nullptr;
  unsigned* ticket = nullptr;
  DevParams* dparams = nullptr;
  DevSplats* dsplats = nullptr;   // inside dparams' allocation, right after the parameters
  // the two diagnostics blocks and the dt slots in one allocation (diag_block_offset)
  double* diag = nullptr;           // the allocation
  int diag_next = 0;                // the block the next diagnostics launch fills (the other is clear)
  int diag_last = 0;                // the block the last one filled
  double* seed_parts = nullptr;
  uint32_t* step_counter = nullptr;   // device copy of step_index for S2D_STEP_RELATCH
  int* err = nullptr;                 // device error word (bounded waits that gave up)
  char* tctab = nullptr;              // tensor-core DFT32 planes + twiddle matrix (fft 'tc-f16')
  int* row_nz = nullptr;              // per ky row: the last row-kernel pass wrote a nonzero PA/PB row
  bool packs_flagged = false;         // PA/PB rows flagged zero were left unwritten
  uchar4* image = nullptr;            // headless render target, grown on demand
  size_t image_px = 0;
  ushort4* dye[3] = {nullptr, nullptr, nullptr};
  // pinned readback staging (copyDiagnostics), laid out as the device block
  double* h_diag = nullptr;
  uint32_t* h_fixed = nullptr;      // inside h_diag's allocation
  float* h_zonal = nullptr;         // inside h_diag's allocation
  float* h_dt = nullptr;            // inside h_base: [dt, speed] of the slot current at the copy
  double* h_base = nullptr;         // the pinned allocation (h_diag etc. point at the copied block)
  cudaEvent_t diag_event = nullptr;
  // pinned upload ring for the per-step parameter and splat blocks: slot i is rewritten
  // only after the copy that last read it has run (upload_ev[i])
  char* h_upload = nullptr;
  cudaEvent_t upload_ev[kUploadSlots] = {};
  int upload_next = 0;
  // host mirror of the JS Solver fields
  DevParams hp{};
  DevSplats hs{};
  bool configured = false;
  // host blocks changed since their last upload (sent together before the next device work)
  bool params_dirty = false, splats_dirty = false;
  int phase = 0, dye_parity = 0, slot = 0;
  uint32_t step_index = 0;
  double sim_time = 0.0;
  bool primed = false, packs_valid = false, reduced_valid = false, disposed = false;
  int read_state = 0;  // 0 idle, 1 copied
  bool latch_pending = false;   // S2D_STEP_RELATCH: the next step's first column kernel latches
  int phys_choice = 0, spec_choice = 0;   // stage-kernel shapes in use (ops->phys / ops->spec)
  std::map<GraphKey, GraphEntry> graphs;
  // instrumentation: event pairs around launches, by kernel class
  bool profiling = false;
  std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> prof_events;
  double prof_ms[S2D_PROF_CLASSES] = {0};
  int prof_cnt[S2D_PROF_CLASSES] = {0};
};

// device block b of the diagnostics allocation: FP64 bins, u32 bins, zonal mean
static double* diag_fp64(s2d_solver* s, int b) {
  return reinterpret_cast<double*>(reinterpret_cast<char*>(s->diag) + diag_block_offset(s->nbins, s->n, b));
}
static uint32_t* diag_u32(s2d_solver* s, int b) { return reinterpret_cast<uint32_t*>(diag_fp64(s, b) + s->nbins + 2); }
static float* diag_zonal(s2d_solver* s, int b) { return reinterpret_cast<float*>(diag_u32(s, b) + s->nbins + 2); }
// point the host views at pinned block b (the one the last copy read)
static void set_host_diag_block(s2d_solver* s, int b) {
  s->h_diag = reinterpret_cast<double*>(reinterpret_cast<char*>(s->h_base) + diag_block_offset(s->nbins, s->n, b));
  s->h_fixed = reinterpret_cast<uint32_t*>(s->h_diag + s->nbins + 2);
  s->h_zonal = reinterpret_cast<float*>(s->h_fixed + s->nbins + 2);
}

// Row-stage variants of a solver: the registered FP32 shapes, plus (last index) the row
// stage on the tensor cores for a tensor-core solver.
static int spec_variants(const s2d_solver* s) {
  return s->ops->n_spec + (s->fft_precision != S2D_FFT_FP32 && s->n == 1024 ? 1 : 0);
}
static bool tc_rows(const s2d_solver* s) {
  return s->fft_precision != S2D_FFT_FP32 && s->n == 1024 && s->spec_choice == s->ops->n_spec;
}

// Stage-kernel shapes chosen by s2d_autotune, per (device, n, FFT precision), shared by
// the solvers created afterwards in this process.
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int>, std::pair<int, int>> g_tuned;
static void tuned_choice(s2d_solver* s) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(std::make_tuple(s->dev, s->n, s->fft_precision));
  if (it == g_tuned.end()) return;
  if (it->second.first < s->ops->n_phys) s->phys_choice = it->second.first;
  if (it->second.second < spec_variants(s)) s->spec_choice = it->second.second;
}
static void remember_choice(s2d_solver* s) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[std::make_tuple(s->dev, s->n, s->fft_precision)] = std::make_pair(s->phys_choice, s->spec_choice);
}

// RAII event pair around the launches of one kernel class (when profiling).
// Inside stream capture the records must be external to become event-record
// nodes of the graph (a plain record there only orders the capture).
struct ProfScope {
  s2d_solver* s;
  int cls;
  cudaEvent_t a = nullptr, b = nullptr;
  static void record(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
    else cudaEventRecord(e, st);
  }
  ProfScope(s2d_solver* s_, int c) : s(s_), cls(c) {
    if (!s->profiling) return;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return;
    record(a, s->stream);
  }
  ~ProfScope() {
    if (!a || !b) return;
    record(b, s->stream);
    s->prof_events.emplace_back(cls, a, b);
  }
};

static int seed_parts_count(int n) { return (n * n + 255) / 256; }

static void free_solver(s2d_solver* s) {
  if (s->diag_stream) cudaStreamSynchronize(s->diag_stream);   // its copies read device memory
  for (auto& kv : s->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    for (auto& ev : kv.second.events) {
      cudaEventDestroy(std::get<1>(ev));
      cudaEventDestroy(std::get<2>(ev));
    }
  }
  s->graphs.clear();
  for (auto& ev : s->prof_events) {
    cudaEventDestroy(std::get<1>(ev));
    cudaEventDestroy(std::get<2>(ev));
  }
  s->prof_events.clear();
  void* dev_ptrs[] = {s->state[0], s->state[1], s->state[2], s->packA, s->packB, s->physZ, s->rhs,
                      s->force, s->vel, s->tw, s->partials, s->ticket, s->dparams, s->diag, s->seed_parts,
                      s->step_counter, s->err, s->tctab, s->row_nz, s->image, s->dye[0], s->dye[1], s->dye[2]};
  for (void* p : dev_ptrs)
    if (p) cudaFree(p);
  void* host_ptrs[] = {s->h_base, s->h_upload};
  for (void* p : host_ptrs)
    if (p) cudaFreeHost(p);
  for (cudaEvent_t ev : {s->diag_event, s->diag_ready, s->diag_done})
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : s->upload_ev)
    if (ev) cudaEventDestroy(ev);
  if (s->diag_stream) cudaStreamDestroy(s->diag_stream);
  if (s->stream) cudaStreamDestroy(s->stream);
}

// host -> device copy of a small per-step block through the pinned upload ring; the
// source may be reused as soon as this returns
static cudaError_t upload(s2d_solver* s, void* dst, const void* src, size_t bytes) {
  const int i = s->upload_next;
  s->upload_next = (i + 1) % kUploadSlots;
  cudaError_t e = cudaEventSynchronize(s->upload_ev[i]);   // the copy that last read slot i
  if (e != cudaSuccess) return e;
  char* slot = s->h_upload + (size_t)i * kUploadSlotBytes;
  std::memcpy(slot, src, bytes);
  e = cudaMemcpyAsync(dst, slot, bytes, cudaMemcpyHostToDevice, s->stream);
  if (e != cudaSuccess) return e;
  return cudaEventRecord(s->upload_ev[i], s->stream);
}

// configure() and setSplats() only update the host blocks; the changed ones go to the
// device in one copy ahead of the next call that enqueues work or reads the device
// (every entry point below except those two and the host-only getters)
static int flush_uploads(s2d_solver* s) {
  if (!s->params_dirty && !s->splats_dirty) return S2D_OK;
  DeviceGuard guard(s->dev);
  char block[kConstBytes];
  std::memcpy(block, &s->hp, sizeof(DevParams));
  std::memcpy(block + sizeof(DevParams), &s->hs, sizeof(DevSplats));
  const size_t lo = s->params_dirty ? 0 : sizeof(DevParams);
  const size_t hi = s->splats_dirty ? kConstBytes : sizeof(DevParams);
  const cudaError_t e = upload(s, reinterpret_cast<char*>(s->dparams) + lo, block + lo, hi - lo);
  if (e != cudaSuccess) return fail(S2D_ERR_CUDA, std::string("parameter upload: ") + cudaGetErrorString(e));
  s->params_dirty = s->splats_dirty = false;
  return S2D_OK;
}

#define S2D_USE_HOST(s)                                                    \
  do {                                                                     \
    if (!(s)) return fail(S2D_ERR_ARG, "null solver handle");              \
    if ((s)->disposed) return fail(S2D_ERR_DESTROYED, "solver destroyed"); \
  } while (0)
static bool stream_capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}
// the main stream waits for the outstanding spectra launch (see s2d_solver::diag_stream)
static int diag_order(s2d_solver* s) {
  if (!s->diag_outstanding) return S2D_OK;
  s->diag_outstanding = false;
  // a caller capturing the main stream into a graph: the graph runs later, after the
  // spectra have finished on the host's clock
  const cudaError_t e = stream_capturing(s->stream) ? cudaEventSynchronize(s->diag_done)
                                                    : cudaStreamWaitEvent(s->stream, s->diag_done, 0);
  return e == cudaSuccess ? S2D_OK : fail(S2D_ERR_CUDA, std::string("diagnostics order: ") + cudaGetErrorString(e));
}
// Every entry point that enqueues device work (or reads the device) flushes the host
// blocks and orders the main stream after the outstanding spectra; the step entry points
// order only where a step may write what the spectra read (diag_order_step), and the
// readback calls, which use the diagnostics stream, do not order.
#define S2D_USE_NOORDER(s)                           \
  do {                                               \
    S2D_USE_HOST(s);                                 \
    if (int rc_ = flush_uploads(s)) return rc_;      \
  } while (0)
#define S2D_USE(s)                                                    \
  do {                                                                \
    S2D_USE_NOORDER(s);                                               \
    if (!(s)->in_step)                                                \
      if (int rc_ = diag_order(s)) return rc_;                        \
  } while (0)
// marks the body of a step call: its inner entry points leave the ordering to it
struct InStep {
  s2d_solver* s;
  explicit InStep(s2d_solver* s_) : s(s_) { ++s->in_step; }
  ~InStep() { --s->in_step; }
};

// ------------------------------------------------------------------ library entry points
extern "C" int s2d_version(void) { return 10000; }

extern "C" const char* s2d_status_string(int st) {
  switch (st) {
    case S2D_OK: return "ok";
    case S2D_NO_DATA: return "no data";
    case S2D_ERR_ARG: return "bad argument";
    case S2D_ERR_UNSUPPORTED_N: return "unsupported grid size";
    case S2D_ERR_CUDA: return "CUDA error";
    case S2D_ERR_DESTROYED: return "use after destroy";
    case S2D_ERR_NAN: return "non-finite input";
    case S2D_ERR_UNREGISTERED: return "buffer was never registered with the FFT";
    case S2D_ERR_NO_DEVICE: return "no usable device";
    default: return "unknown status";
  }
}

extern "C" const char* s2d_last_error(void) { return g_last_error.c_str(); }

extern "C" int s2d_radix_schedule(int n, int* stages, int* has_radix2) {
  if (!radix_ok(n, stages, has_radix2))
    return fail(S2D_ERR_UNSUPPORTED_N, "grid size " + std::to_string(n) + " must be 4^a or 2 * 4^a");
  return S2D_OK;
}

extern "C" int s2d_supported_grids(int* out, int capacity, int* count) {
  if (!count) return fail(S2D_ERR_ARG, "count is null");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(S2D_ERR_NO_DEVICE, "no CUDA device");
  int smem_optin = 0;
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  int c = 0;
  for (int n = S2D_MIN_N; n <= S2D_MAX_N; n *= 2) {
    const NOps* o = ops_for(n);
    if (!o) continue;
    const size_t need_smem = o->a_smem > o->b_smem ? o->a_smem : o->b_smem;
    const size_t need_mem = (size_t)n * n * 8 * 10;   // 3 states, 6 work buffers, velocity
    if (need_smem > (size_t)smem_optin || need_mem > total_b) continue;
    if (out && c < capacity) out[c] = n;
    ++c;
  }
  *count = c;
  return S2D_OK;
}

// One axis of one tile of k_dye_fused: the tile starts at texel t0 and has T texels; the
// backward / forward / source regions have W1 / W2 / W3 texels and the velocity window
// vw cells, with the origins dye_cta_setup computes (src_lo: the source window's extra
// texels below its halo).  A trace shorter than one texel from texel x has its bilinear
// footprint's first texel at x - 1 or x, and its midpoint (half the displacement) reads
// the velocity at a coordinate (x + 0.5 + d) n/m - 0.5 with |d| <= 1/2.
static const char* dye_axis_check(int n, int m, int t0, int T, int W1, int W2, int W3, int src_lo, int vw) {
  const long s_org = t0 - src_lo, f_org = t0 - 2 * kDyeLo, b_org = t0 - kDyeLo;
  const long v_org = (long)floorf(((float)(t0 - 2 * kDyeLo - 1) + 0.5f) * (float)n / (float)m - 0.5f) - 1;
  // slot of texel (or cell) t in a window at origin org holding w entries of a periodic
  // axis of len: its lookup reads this slot and the next
  auto fits = [](long t, long org, int w, int len) {
    const long d = ((t - org) % len + len) % len;
    return d + 1 < w;
  };
  auto footprints_in = [&](long x, long org, int w) { return fits(x - 1, org, w, m) && fits(x, org, w, m); };
  auto velocity_in = [&](long x) {
    for (int d = -1; d <= 1; ++d) {   // d / 2 texels: the midpoint extremes and the centre
      const double g = ((double)x + 0.5 + 0.5 * d) * (double)n / (double)m - 0.5;
      if (!fits((long)std::floor(g), v_org, vw, n)) return false;
    }
    return true;
  };
  for (long x = f_org; x < f_org + W2; ++x) {
    if (!footprints_in(x, s_org, W3)) return "forward footprint outside the source window";
    if (!velocity_in(x)) return "forward-region trace outside the velocity window";
  }
  for (long x = b_org; x < b_org + W1; ++x)
    if (!footprints_in(x, f_org, W2)) return "backward footprint outside the forward window";
  for (long x = t0; x < t0 + T; ++x) {
    if (!footprints_in(x, s_org, W3)) return "corrected footprint outside the source window";
    if (!footprints_in(x, b_org, W1)) return "corrected footprint outside the backward window";
  }
  return nullptr;
}

template <int TX> static int dye_fast_path_check_tx(int n, int m) {
  using G = DyeGeom<TX>;
  for (int t0 = 0; t0 < m; t0 += TX)
    if (const char* why = dye_axis_check(n, m, t0, TX, G::W1X, G::W2X, G::W3X, 3 * kDyeLo + 1, G::vel_x(n, m)))
      return fail(S2D_ERR_ARG, std::string("x tile at ") + std::to_string(t0) + ": " + why);
  for (int t0 = 0; t0 < m; t0 += G::TY)
    if (const char* why = dye_axis_check(n, m, t0, G::TY, G::W1Y, G::W2Y, G::W3Y, 3 * kDyeLo, G::vel_y(n, m)))
      return fail(S2D_ERR_ARG, std::string("y tile at ") + std::to_string(t0) + ": " + why);
  return S2D_OK;
}

extern "C" int s2d_dye_fast_path_check(int n, int dye_scale) {
  if (n < S2D_MIN_N || n > S2D_MAX_N || (n & (n - 1)) != 0) return fail(S2D_ERR_UNSUPPORTED_N, "n");
  if (dye_scale != 1 && dye_scale != 2 && dye_scale != 4) return fail(S2D_ERR_ARG, "dye_scale must be 1, 2 or 4");
  const int m = n * dye_scale;
  return dye_wide_tile(n, m) ? dye_fast_path_check_tx<64>(n, m) : dye_fast_path_check_tx<32>(n, m);
}

static int table_prelude(int n) {
  if (n < 2 || n > (1 << 16) || (n & (n - 1))) return fail(S2D_ERR_UNSUPPORTED_N, "size must be a power of two");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(S2D_ERR_NO_DEVICE, "no CUDA device");
  return check_device(dev);
}

extern "C" int s2d_digit_reverse_table(int n, uint32_t* out) {
  int st = 0, r2 = 0;
  if (!out) return fail(S2D_ERR_ARG, "out is null");
  if (!radix_ok(n, &st, &r2)) return fail(S2D_ERR_UNSUPPORTED_N, "size must be 4^a or 2 * 4^a");
  if (int rc = table_prelude(n)) return rc;
  uint32_t* d = nullptr;
  S2D_CUDA(cudaMalloc(&d, sizeof(uint32_t) * n));
  k_digit_reverse<<<(n + 255) / 256, 256>>>(d, n, st, r2);
  cudaError_t e = cudaMemcpy(out, d, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(S2D_ERR_CUDA, cudaGetErrorString(e));
  return S2D_OK;
}

extern "C" int s2d_wavenumber_table(int n, float* out) {
  if (!out) return fail(S2D_ERR_ARG, "out is null");
  if (int rc = table_prelude(n)) return rc;
  float* d = nullptr;
  S2D_CUDA(cudaMalloc(&d, sizeof(float) * n));
  k_wavenumbers<<<(n + 255) / 256, 256>>>(d, n);
  cudaError_t e = cudaMemcpy(out, d, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(S2D_ERR_CUDA, cudaGetErrorString(e));
  return S2D_OK;
}

extern "C" int s2d_dealias_mask_table(int n, uint8_t* out) {
  if (!out) return fail(S2D_ERR_ARG, "out is null");
  if (int rc = table_prelude(n)) return rc;
  uint8_t* d = nullptr;
  const size_t cells = (size_t)n * n;
  S2D_CUDA(cudaMalloc(&d, cells));
  k_mask_table<<<(unsigned)((cells + 255) / 256), 256>>>(d, n);
  cudaError_t e = cudaMemcpy(out, d, cells, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(S2D_ERR_CUDA, cudaGetErrorString(e));
  return S2D_OK;
}

// ------------------------------------------------------------------ lifecycle
// ------------------------------------------------------------------ tensor-core kernels by precision
template <class P> static cudaError_t tc_attrs() {
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) { if (r != cudaSuccess && e == cudaSuccess) e = r; };
  const int smem = tc::kTcSmem;
  chk(cudaFuncSetAttribute(tc::k_fft_tc<0, -1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  chk(cudaFuncSetAttribute(tc::k_fft_tc<0, +1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  chk(cudaFuncSetAttribute(tc::k_fft_tc<1, -1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  chk(cudaFuncSetAttribute(tc::k_fft_tc<1, +1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  chk(cudaFuncSetAttribute(tc::k_phys_cols_tc2<0, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_phys_cols_tc2<1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_phys_cols_tc2<2, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_spec_rows_tc2<-1, false, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_spec_rows_tc2<0, false, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_spec_rows_tc2<1, false, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_spec_rows_tc2<2, false, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_spec_rows_tc2<0, true, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_spec_rows_tc2<1, true, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  chk(cudaFuncSetAttribute(tc::k_spec_rows_tc2<2, true, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kC2Smem));
  return e;
}
template <class P> static void tc_fft2_launch(float2* buf, int sign, const char* tab, int* err, cudaStream_t st) {
  const dim3 g(1024 / tc::kTcLines), b(tc::kTcThreads);
  if (sign < 0) {
    tc::k_fft_tc<0, -1, P><<<g, b, tc::kTcSmem, st>>>(buf, tab, err);
    tc::k_fft_tc<1, -1, P><<<g, b, tc::kTcSmem, st>>>(buf, tab, err);
  } else {
    tc::k_fft_tc<0, +1, P><<<g, b, tc::kTcSmem, st>>>(buf, tab, err);
    tc::k_fft_tc<1, +1, P><<<g, b, tc::kTcSmem, st>>>(buf, tab, err);
  }
}
template <class P> static void tc_cols_launch(int mode, const PhysArgs& a, const char* tab, int* err, cudaStream_t st) {
  const dim3 g(tc::kC2Grid), b(tc::kC2Threads);
  if (mode == 0) tc::k_phys_cols_tc2<0, P><<<g, b, tc::kC2Smem, st>>>(a, tab, err);
  else if (mode == 1) tc::k_phys_cols_tc2<1, P><<<g, b, tc::kC2Smem, st>>>(a, tab, err);
  else tc::k_phys_cols_tc2<2, P><<<g, b, tc::kC2Smem, st>>>(a, tab, err);
}
// the row stage on the tensor cores: mode -1 = prime (pack wcur only), 0..2 = RK stage
template <class P> static void tc_rows_launch(int mode, bool ptr, const SpecArgs& a, const char* tab, cudaStream_t st) {
  const dim3 g(512 / tc::kC2Wg), b(tc::kC2Threads);
  const int sm = tc::kC2Smem;
  if (mode < 0) tc::k_spec_rows_tc2<-1, false, P><<<g, b, sm, st>>>(a, tab);
  else if (!ptr) {
    if (mode == 0) tc::k_spec_rows_tc2<0, false, P><<<g, b, sm, st>>>(a, tab);
    else if (mode == 1) tc::k_spec_rows_tc2<1, false, P><<<g, b, sm, st>>>(a, tab);
    else tc::k_spec_rows_tc2<2, false, P><<<g, b, sm, st>>>(a, tab);
  } else {
    if (mode == 0) tc::k_spec_rows_tc2<0, true, P><<<g, b, sm, st>>>(a, tab);
    else if (mode == 1) tc::k_spec_rows_tc2<1, true, P><<<g, b, sm, st>>>(a, tab);
    else tc::k_spec_rows_tc2<2, true, P><<<g, b, sm, st>>>(a, tab);
  }
}
static bool is_tc(const s2d_solver* s) { return s->fft_precision != S2D_FFT_FP32; }
// the row stage with the solver's chosen variant
static void run_spec(s2d_solver* s, int mode, bool ptr, const SpecArgs& a) {
  if (tc_rows(s)) {
    if (s->fft_precision == S2D_FFT_TC_BF16) tc_rows_launch<tc::PrecBF16>(mode, ptr, a, s->tctab, s->stream);
    else tc_rows_launch<tc::PrecF16>(mode, ptr, a, s->tctab, s->stream);
  } else {
    s->ops->spec[s->spec_choice].run(mode, ptr, a, s->stream);
  }
}

extern "C" int s2d_create(int n, int dye_scale, int fft_precision, int device, s2d_solver** out) {
  if (!out) return fail(S2D_ERR_ARG, "out is null");
  *out = nullptr;
  if (!radix_ok(n, nullptr, nullptr) && !(n >= S2D_MIN_N && (n & (n - 1)) == 0))
    return fail(S2D_ERR_UNSUPPORTED_N, "grid size " + std::to_string(n) + " must be a power of two");
  const NOps* ops = ops_for(n);
  if (!ops) return fail(S2D_ERR_UNSUPPORTED_N, "grid size " + std::to_string(n) + " outside 32..4096");
  // the dye grid must be a power of two (wrapped texel indices, exact texel centres): the
  // reference offers dyeScale 1 and 2 (main.js:196); 4 is accepted as well
  if (dye_scale != 1 && dye_scale != 2 && dye_scale != 4)
    return fail(S2D_ERR_ARG, "dye_scale must be 1, 2 or 4");
  if (fft_precision != S2D_FFT_FP32 && fft_precision != S2D_FFT_TC_F16 && fft_precision != S2D_FFT_TC_BF16)
    return fail(S2D_ERR_ARG, "unknown FFT arithmetic (S2D_FFT_FP32, S2D_FFT_TC_F16, S2D_FFT_TC_BF16)");
  if (fft_precision != S2D_FFT_FP32 && n != 1024 && !tc::tc_lines_supported(n))
    return fail(S2D_ERR_UNSUPPORTED_N, "the tensor-core FFT is built for N = 256, 512, 1024, 2048, 4096");
  if (int rc = check_device(device)) return rc;
  DeviceGuard guard(device);
  s2d_solver* s = new s2d_solver();
  s->dev = device;
  s->n = n;
  s->m = n * dye_scale;
  s->dye_scale = dye_scale;
  s->nbins = n / 2 + 1;
  s->fft_precision = fft_precision;
  s->ops = ops;
  tuned_choice(s);
  const size_t cbytes = (size_t)n * n * sizeof(float2);
  const size_t dbytes = (size_t)s->m * s->m * sizeof(ushort4);
  auto bail = [&](cudaError_t e, const char* what) {
    free_solver(s);
    delete s;
    return fail(S2D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  cudaError_t e;
#define TRY(call, what)            \
  if ((e = (call)) != cudaSuccess) \
    return bail(e, what);
  // the step work ahead of the diagnostics spectra when both have CTAs waiting for an SM
  int prio_least = 0, prio_greatest = 0;
  TRY(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest), "stream priorities");
  TRY(cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, prio_greatest), "stream");
  TRY(cudaStreamCreateWithPriority(&s->diag_stream, cudaStreamNonBlocking, prio_least), "diagnostics stream");
  TRY(cudaEventCreateWithFlags(&s->diag_event, cudaEventDisableTiming), "event");
  TRY(cudaEventCreateWithFlags(&s->diag_ready, cudaEventDisableTiming), "event");
  TRY(cudaEventCreateWithFlags(&s->diag_done, cudaEventDisableTiming), "event");
  for (int i = 0; i < 3; ++i) TRY(cudaMalloc(&s->state[i], cbytes), "state");
  TRY(cudaMalloc(&s->packA, cbytes), "packA");
  TRY(cudaMalloc(&s->packB, cbytes), "packB");
  TRY(cudaMalloc(&s->physZ, cbytes), "physZ");
  TRY(cudaMalloc(&s->rhs, cbytes), "rhs");
  TRY(cudaMalloc(&s->force, cbytes), "force");
  TRY(cudaMalloc(&s->vel, cbytes), "vel");
  TRY(cudaMalloc(&s->tw, sizeof(float2) * n), "twiddles");
  // column-kernel grids are at most n CTAs in every registered shape
  const int nparts = std::max(std::max(n, 256), seed_parts_count(n));
  TRY(cudaMalloc(&s->partials, sizeof(float) * nparts), "partials");
  TRY(cudaMalloc(&s->ticket, sizeof(unsigned)), "ticket");
  TRY(cudaMalloc(&s->row_nz, sizeof(int) * n), "row flags");
  TRY(cudaMalloc(&s->dparams, kConstBytes), "params");
  s->dsplats = reinterpret_cast<DevSplats*>(reinterpret_cast<char*>(s->dparams) + sizeof(DevParams));
  TRY(cudaMalloc(&s->diag, diag_alloc_bytes(s->nbins, n)), "diag");
  TRY(cudaMemsetAsync(s->diag, 0, diag_alloc_bytes(s->nbins, n), s->stream), "memset");   // both blocks clear
  s->dtbuf = reinterpret_cast<float*>(reinterpret_cast<char*>(s->diag) + diag_dt_offset(s->nbins, n));
  TRY(cudaMalloc(&s->seed_parts, sizeof(double) * seed_parts_count(n)), "seed partials");
  TRY(cudaMalloc(&s->step_counter, sizeof(uint32_t)), "step counter");
  TRY(cudaMalloc(&s->err, sizeof(int)), "error word");
  TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->stream), "memset");
  TRY(cudaMemsetAsync(s->step_counter, 0, sizeof(uint32_t), s->stream), "memset");
  for (int i = 0; i < 3; ++i) TRY(cudaMalloc(&s->dye[i], dbytes), "dye");
  TRY(cudaMallocHost(&s->h_base, diag_alloc_bytes(s->nbins, n)), "pinned diag");
  std::memset(s->h_base, 0, diag_alloc_bytes(s->nbins, n));
  s->h_dt = reinterpret_cast<float*>(reinterpret_cast<char*>(s->h_base) + diag_dt_offset(s->nbins, n));   // [dt, speed]
  set_host_diag_block(s, 0);
  TRY(cudaMallocHost(&s->h_upload, kUploadSlotBytes * kUploadSlots), "pinned upload ring");
  for (cudaEvent_t& ev : s->upload_ev) TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
  TRY(set_all_attrs(*ops), "kernel attributes");
  if (dye_wide_tile(n, s->m))
    TRY(cudaFuncSetAttribute(k_dye_fused<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)DyeGeom<64>::smem(n, s->m)), "dye kernel attributes");
  TRY(cudaFuncSetAttribute(k_dye_fused<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)DyeGeom<32>::smem(n, s->m)), "dye kernel attributes");
  if (fft_precision == S2D_FFT_TC_F16 && n == 1024) TRY(tc_attrs<tc::PrecF16>(), "tensor-core kernel attributes");
  if (fft_precision == S2D_FFT_TC_BF16 && n == 1024) TRY(tc_attrs<tc::PrecBF16>(), "tensor-core kernel attributes");
  if (fft_precision != S2D_FFT_FP32 && n != 1024)
    TRY(tc::tc_lines_attrs(n, fft_precision == S2D_FFT_TC_BF16), "tensor-core kernel attributes");
  // zero everything the reference's fresh buffers hold as zero
  for (int i = 0; i < 3; ++i) TRY(cudaMemsetAsync(s->state[i], 0, cbytes, s->stream), "memset");
  TRY(cudaMemsetAsync(s->packA, 0, cbytes, s->stream), "memset");
  TRY(cudaMemsetAsync(s->packB, 0, cbytes, s->stream), "memset");
  TRY(cudaMemsetAsync(s->physZ, 0, cbytes, s->stream), "memset");
  TRY(cudaMemsetAsync(s->rhs, 0, cbytes, s->stream), "memset");
  TRY(cudaMemsetAsync(s->force, 0, cbytes, s->stream), "memset");
  TRY(cudaMemsetAsync(s->vel, 0, cbytes, s->stream), "memset");
  TRY(cudaMemsetAsync(s->dtbuf, 0, sizeof(float) * 4, s->stream), "memset");
  TRY(cudaMemsetAsync(s->ticket, 0, sizeof(unsigned), s->stream), "memset");
  TRY(cudaMemsetAsync(s->partials, 0, sizeof(float) * nparts, s->stream), "memset");
  for (int i = 0; i < 3; ++i) TRY(cudaMemsetAsync(s->dye[i], 0, dbytes, s->stream), "memset");
  k_twiddles<<<(n + 255) / 256, 256, 0, s->stream>>>(s->tw, n);
  TRY(cudaGetLastError(), "twiddle kernel");
  if (fft_precision != S2D_FFT_FP32 && n == 1024) {
    TRY(cudaMalloc(&s->tctab, tc::kTabBytes), "tensor-core tables");
    if (fft_precision == S2D_FFT_TC_BF16) tc::k_tc_tables<tc::PrecBF16><<<1, 256, 0, s->stream>>>(s->tctab, s->tw);
    else tc::k_tc_tables<tc::PrecF16><<<1, 256, 0, s->stream>>>(s->tctab, s->tw);
    TRY(cudaGetLastError(), "tensor-core table kernel");
  } else if (fft_precision != S2D_FFT_FP32) {
    TRY(cudaMalloc(&s->tctab, tc::tc_lines_table_bytes(n)), "tensor-core tables");
    tc::tc_lines_tables(n, fft_precision == S2D_FFT_TC_BF16, s->tctab, s->tw, s->stream);
    TRY(cudaGetLastError(), "tensor-core table kernel");
  }
  // an unconfigured solver has all-zero parameters apart from the grid constants
  s->hp = DevParams{};
  s->hp.n = n;
  s->hp.kcut = (float)(n / 3.0);
  s->hp.force_norm = (float)(0.01 * n * n);
  s->hp.dx = (float)(2.0 * M_PI / n);
  s->hs = DevSplats{};
  s->params_dirty = s->splats_dirty = true;
  if (int rc = flush_uploads(s)) {
    free_solver(s);
    delete s;
    return rc;
  }
  TRY(cudaStreamSynchronize(s->stream), "create sync");
#undef TRY
  *out = s;
  return S2D_OK;
}

extern "C" int s2d_destroy(s2d_solver* s) {
  if (!s) return fail(S2D_ERR_ARG, "null solver handle");
  DeviceGuard guard(s->dev);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->diag_stream) cudaStreamSynchronize(s->diag_stream);
  s->disposed = true;
  free_solver(s);
  delete s;
  return S2D_OK;
}

extern "C" int s2d_get_info(s2d_solver* s, s2d_info* out) {
  S2D_USE_HOST(s);
  if (!out) return fail(S2D_ERR_ARG, "out is null");
  out->n = s->n;
  out->m = s->m;
  out->nbins = s->nbins;
  out->phase = s->phase;
  out->dye_parity = s->dye_parity;
  out->step_index = s->step_index;
  out->primed = s->primed ? 1 : 0;
  out->fft_precision = s->fft_precision;
  out->nu_h = s->hp.nu_h;
  out->sim_time = s->sim_time;
  return S2D_OK;
}

extern "C" int s2d_set_phase(s2d_solver* s, int phase, int dye_parity) {
  S2D_USE_HOST(s);
  if (phase < 0 || phase > 2 || dye_parity < 0 || dye_parity > 1) return fail(S2D_ERR_ARG, "phase out of range");
  if (phase != s->phase) {
    // the next step writes other ring buffers: none may be one the outstanding spectra read
    DeviceGuard guard(s->dev);
    if (int rc = diag_order(s)) return rc;
    s->packs_valid = false;
  }
  s->phase = phase;
  s->dye_parity = dye_parity;
  return S2D_OK;
}

extern "C" int s2d_set_sim_time(s2d_solver* s, double t) {
  S2D_USE_HOST(s);
  s->sim_time = t;
  return S2D_OK;
}

extern "C" int s2d_get_stream(s2d_solver* s, void** stream) {
  S2D_USE_HOST(s);
  if (!stream) return fail(S2D_ERR_ARG, "out is null");
  *stream = (void*)s->stream;
  return S2D_OK;
}

// reports (and clears) a bounded device-side wait that gave up since the last check
static int check_device_error(s2d_solver* s) {
  int h = 0;
  S2D_CUDA(cudaMemcpyAsync(&h, s->err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  if (h) {
    cudaMemsetAsync(s->err, 0, sizeof(int), s->stream);
    return fail(S2D_ERR_CUDA, "a bounded device-side wait gave up (site " + std::to_string(h) +
                                  "); results of the work enqueued since the last check are invalid");
  }
  return S2D_OK;
}

// One CTA whose barrier expects 16 bytes that no copy ever delivers: its bounded wait
// gives up after limit_ns, records site 5 in the error word and the kernel returns.
// Nothing is in flight when it exits (no copy was issued), so the context stays usable.
static __global__ void k_wait_probe(int* err, unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16u);
  __syncthreads();
  mbar_wait_bounded(&bar, 0u, err, 5, limit_ns);
}

extern "C" int s2d_probe_wait_timeout(s2d_solver* s, unsigned long long limit_ns) {
  S2D_USE(s);
  if (limit_ns == 0 || limit_ns > 1000000000ull) return fail(S2D_ERR_ARG, "limit_ns must be in 1..1e9");
  DeviceGuard guard(s->dev);
  k_wait_probe<<<1, 32, 0, s->stream>>>(s->err, limit_ns);
  S2D_CUDA(cudaGetLastError());
  return S2D_OK;
}

extern "C" int s2d_synchronize(s2d_solver* s) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  S2D_CUDA(cudaStreamSynchronize(s->diag_stream));
  return check_device_error(s);
}

// ------------------------------------------------------------------ parameters
extern "C" int s2d_configure(s2d_solver* s, const s2d_params* p) {
  S2D_USE_HOST(s);
  if (!p) return fail(S2D_ERR_ARG, "params is null");
  if (p->hyper_p < 0 || p->hyper_p > 16) return fail(S2D_ERR_ARG, "hyperP must be in 0..16");
  const double kcut = s->n / 3.0;
  DevParams& h = s->hp;
  h.beta = p->beta;
  h.mu = p->drag;
  h.nu_h = p->viscosity > 0 ? (float)(p->viscosity / std::pow(kcut, 2.0 * p->hyper_p)) : 0.f;
  h.hyper_p = p->hyper_p;
  h.force_amp = p->force_amp;
  h.force_k = p->force_k;
  h.force_width = p->force_width;
  h.step_index = s->step_index;    // latched once per configure (solver.js:316)
  h.dx = (float)(2.0 * M_PI / s->n);
  h.cfl = p->cfl;
  h.dt_min = p->dt_min;
  h.dt_max = p->dt_max;
  h.dye_fade = p->dye_fade;
  h.kcut = (float)kcut;
  h.force_norm = (float)(0.01 * s->n * s->n);
  h.n = s->n;
  s->params_dirty = true;   // uploaded with the next device work (flush_uploads)
  s->configured = true;
  return S2D_OK;
}

extern "C" int s2d_set_splats(s2d_solver* s, const s2d_splat* list, int count) {
  S2D_USE_HOST(s);
  if (count < 0 || (count > 0 && !list)) return fail(S2D_ERR_ARG, "bad splat list");
  const int c = count < S2D_MAX_SPLATS ? count : S2D_MAX_SPLATS;   // Math.min (solver.js:327)
  s->hs = DevSplats{};
  s->hs.count = c;
  for (int i = 0; i < c; ++i) {
    const s2d_splat& a = list[i];
    DevSplat& d = s->hs.items[i];
    d.x = a.x; d.y = a.y; d.vx = a.dx; d.vy = a.dy;
    d.r = a.color[0]; d.g = a.color[1]; d.b = a.color[2];
    d.radius = a.radius; d.amp = a.amp; d.dye_amp = a.dye_amp;
  }
  s->splats_dirty = true;   // uploaded with the next device work (flush_uploads)
  return S2D_OK;
}

// ------------------------------------------------------------------ internal enqueue helpers
static inline unsigned cells_grid(int n) { return (unsigned)(((size_t)n * n + 255) / 256); }

static int enqueue_fft2(s2d_solver* s, float2* buf, int sign) {
  if (is_tc(s)) {
    // tensor-core DFT-GEMM passes: 8 lines of 1024 per CTA, or the generic N1 x N2 form
    if (s->n != 1024)
      tc::tc_lines_fft2(s->n, s->fft_precision == S2D_FFT_TC_BF16, buf, sign, s->tctab, s->tw, s->err, s->stream);
    else if (s->fft_precision == S2D_FFT_TC_BF16) tc_fft2_launch<tc::PrecBF16>(buf, sign, s->tctab, s->err, s->stream);
    else tc_fft2_launch<tc::PrecF16>(buf, sign, s->tctab, s->err, s->stream);
    S2D_LAUNCHED();
    return S2D_OK;
  }
  s->ops->fft_rows(sign, buf, s->tw, s->stream);
  S2D_LAUNCHED();
  s->ops->fft_cols(sign, buf, s->tw, s->stream);
  S2D_LAUNCHED();
  return S2D_OK;
}

static float* dt_slot(s2d_solver* s, int slot) { return s->dtbuf + 2 * slot; }

// prime packs from state[phase]: PA/PB = FFT_x^-1 of the scaled packs
static int enqueue_pack_prime(s2d_solver* s) {
  SpecArgs a{};
  a.wcur = s->state[s->phase];
  a.pa = s->packA;
  a.pb = s->packB;
  a.dt = dt_slot(s, s->slot);
  a.params = s->dparams;
  a.tw = s->tw;
  a.err = s->err;
  a.row_nz = s->row_nz;
  run_spec(s, -1, false, a);
  S2D_LAUNCHED();
  s->packs_flagged = true;
  s->packs_valid = true;
  return S2D_OK;
}

// make the rows the row kernel skipped (flagged all zero) explicit zeros, before anything
// other than the fused stage kernels reads or writes the packs
static int materialize_packs(s2d_solver* s) {
  if (!s->packs_flagged) return S2D_OK;
  k_zero_flagged_rows<<<cells_grid(s->n), 256, 0, s->stream>>>(s->packA, s->packB, s->row_nz, s->n);
  S2D_LAUNCHED();
  s->packs_flagged = false;
  return S2D_OK;
}

static PhysArgs phys_args(s2d_solver* s, int reduce) {
  PhysArgs a{};
  a.pa = s->packA;
  a.pb = s->packB;
  a.z = s->physZ;
  a.vel = s->vel;
  a.partials = s->partials;
  a.ticket = s->ticket;
  a.dt_out = dt_slot(s, s->slot ^ 1);
  a.params = s->dparams;
  a.tw = s->tw;
  a.reduce = reduce;
  a.row_nz = s->row_nz;
  return a;
}

// the physical-column stage: tensor-core y-transforms when the solver was created
// with S2D_FFT_TC_F16 / S2D_FFT_TC_BF16 (1024^2 only), else the FP32 whole-line kernel
static void enqueue_phys_cols(s2d_solver* s, int mode, const PhysArgs& a) {
  if (is_tc(s)) {
    if (s->fft_precision == S2D_FFT_TC_BF16) tc_cols_launch<tc::PrecBF16>(mode, a, s->tctab, s->err, s->stream);
    else tc_cols_launch<tc::PrecF16>(mode, a, s->tctab, s->err, s->stream);
  } else {
    s->ops->phys[s->phys_choice].run(mode, a, s->stream);
  }
}

extern "C" int s2d_encode_reduce(s2d_solver* s);

// Tensor-core solvers at the sizes without fused tensor-core stage kernels (N != 1024) run
// the reference's per-stage order (solver.js:488-521): velocity pack, two inverse 2D
// transforms, products, forward transform, assemble, RK3 update -- with every 2D transform
// on the tensor cores (s2d_tc_lines.cu) and the pointwise stages on the CUDA cores.
static bool tc_unfused(const s2d_solver* s) { return is_tc(s) && s->n != 1024; }

// velocity (and the packs' physical fields) of state `idx` through the unfused stages
static int enqueue_unfused_velocity(s2d_solver* s, int idx) {
  const unsigned g = cells_grid(s->n);
  k_velocity_pack<<<g, 256, 0, s->stream>>>(s->state[idx], s->packA, s->packB, s->n);
  S2D_LAUNCHED();
  if (int rc = enqueue_fft2(s, s->packA, +1)) return rc;
  if (int rc = enqueue_fft2(s, s->packB, +1)) return rc;
  k_nl_pack<<<g, 256, 0, s->stream>>>(s->packA, s->packB, s->physZ, s->vel, s->n);
  S2D_LAUNCHED();
  return S2D_OK;
}

static int enqueue_unfused_step(s2d_solver* s, bool ptr) {
  if (s->latch_pending) {
    k_latch_step<<<1, 1, 0, s->stream>>>(s->dparams, s->step_counter);
    S2D_LAUNCHED();
    s->latch_pending = false;
  }
  const int p = s->phase;
  const unsigned g = cells_grid(s->n);
  const float* dt = dt_slot(s, s->slot);
  for (int st = 0; st < 3; ++st) {
    if (int rc = enqueue_unfused_velocity(s, (p + st) % 3)) return rc;
    if (int rc = enqueue_fft2(s, s->physZ, -1)) return rc;
    k_assemble<<<g, 256, 0, s->stream>>>(s->physZ, ptr ? s->force : nullptr, dt, s->dparams, s->rhs, s->n);
    S2D_LAUNCHED();
    float2* w0 = s->state[p];
    float2* wc = s->state[(p + st) % 3];
    float2* wo = s->state[(p + (st == 1 ? 2 : 1)) % 3];
    if (st == 0) k_rk3<0><<<g, 256, 0, s->stream>>>(w0, wc, wo, s->rhs, dt, s->dparams, s->n);
    else if (st == 1) k_rk3<1><<<g, 256, 0, s->stream>>>(w0, wc, wo, s->rhs, dt, s->dparams, s->n);
    else k_rk3<2><<<g, 256, 0, s->stream>>>(w0, wc, wo, s->rhs, dt, s->dparams, s->n);
    S2D_LAUNCHED();
  }
  s->reduced_valid = false;   // the CFL reduction runs as its own two launches
  s->packs_valid = false;
  s->packs_flagged = false;
  s->phase = (p + 1) % 3;
  s->step_index += 1;
  return S2D_OK;
}

extern "C" int s2d_encode_prime(s2d_solver* s) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  if (tc_unfused(s)) {
    if (int rc = materialize_packs(s)) return rc;
    if (int rc = enqueue_unfused_velocity(s, s->phase)) return rc;
    s->reduced_valid = false;
    if (int rc = s2d_encode_reduce(s)) return rc;
    s->primed = true;
    return S2D_OK;
  }
  if (int rc = enqueue_pack_prime(s)) return rc;
  PhysArgs a = phys_args(s, 1);
  enqueue_phys_cols(s, 0, a);
  S2D_LAUNCHED();
  s->reduced_valid = true;
  if (int rc = s2d_encode_reduce(s)) return rc;
  s->primed = true;
  return S2D_OK;
}

extern "C" int s2d_encode_step(s2d_solver* s) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  if (!s->packs_valid && !tc_unfused(s))
    if (int rc = enqueue_pack_prime(s)) return rc;
  const bool ptr = s->hs.count > 0;
  if (ptr) {
    ProfScope ps(s, S2D_PROF_FORCE);
    k_pointer_force<<<cells_grid(s->n), 256, 0, s->stream>>>(s->force, s->dsplats, s->n);
    S2D_LAUNCHED();
    if (int rc = enqueue_fft2(s, s->force, -1)) return rc;
  }
  if (tc_unfused(s)) {
    if (int rc = materialize_packs(s)) return rc;
    return enqueue_unfused_step(s, ptr);
  }
  const int p = s->phase;
  for (int st = 0; st < 3; ++st) {
    {
      ProfScope ps(s, S2D_PROF_PHYS_COLS);
      PhysArgs pa = phys_args(s, st == 2 ? 1 : 0);
      if (st == 0 && s->latch_pending) {
        pa.latch = s->dparams;
        pa.counter = s->step_counter;
        s->latch_pending = false;
      }
      enqueue_phys_cols(s, st == 2 ? 2 : 1, pa);
      S2D_LAUNCHED();
    }
    ProfScope ps(s, S2D_PROF_SPEC_ROWS);
    SpecArgs a{};
    a.z = s->physZ;
    a.w0 = s->state[p];
    a.wcur = s->state[(p + st) % 3];
    a.wout = s->state[(p + (st == 1 ? 2 : 1)) % 3];
    a.fptr = ptr ? s->force : nullptr;
    a.pa = s->packA;
    a.pb = s->packB;
    a.dt = dt_slot(s, s->slot);
    a.params = s->dparams;
    a.tw = s->tw;
    a.stochastic = s->hp.force_amp > 0.f ? 1 : 0;
    a.err = s->err;
    a.row_nz = s->row_nz;
    run_spec(s, st, ptr, a);
    S2D_LAUNCHED();
    s->packs_flagged = true;
  }
  s->reduced_valid = true;
  s->packs_valid = true;
  s->phase = (p + 1) % 3;
  s->step_index += 1;
  return S2D_OK;
}

static uint2* tex(s2d_solver* s, int i) { return reinterpret_cast<uint2*>(s->dye[i]); }

// encodeDye (solver.js:523-536) as one fused launch: forward, backward and
// corrected passes of a tile computed from on-chip halos (s2d_dye.cuh)
extern "C" int s2d_encode_dye(s2d_solver* s) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  const int p = s->dye_parity, m = s->m;
  ProfScope ps(s, S2D_PROF_DYE);
  if (dye_wide_tile(s->n, m)) {
    using G = DyeGeom<64>;
    k_dye_fused<64><<<dim3(m / 64, m / G::TY), G::THREADS, G::smem(s->n, m), s->stream>>>(
        s->vel, tex(s, p), tex(s, 1 - p), dt_slot(s, s->slot), s->dparams, s->dsplats, s->n, m);
  } else {
    using G = DyeGeom<32>;
    k_dye_fused<32><<<dim3(m / 32, m / G::TY), G::THREADS, G::smem(s->n, m), s->stream>>>(
        s->vel, tex(s, p), tex(s, 1 - p), dt_slot(s, s->slot), s->dparams, s->dsplats, s->n, m);
  }
  S2D_LAUNCHED();
  s->dye_parity = 1 - p;
  return S2D_OK;
}

// the reference's three dispatches advect_fwd, advect_back, advect_corr (solver.js:523-536)
extern "C" int s2d_encode_dye_passes(s2d_solver* s) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  const int p = s->dye_parity, m = s->m;
  const dim3 blk(16, 16), grd((m + 15) / 16, (m + 15) / 16);
  const float* dt = dt_slot(s, s->slot);
  ProfScope ps(s, S2D_PROF_DYE);
  k_dye_advect<<<grd, blk, 0, s->stream>>>(s->vel, tex(s, p), tex(s, 1 - p), dt, 1.f, s->n, m);
  S2D_LAUNCHED();
  k_dye_advect<<<grd, blk, 0, s->stream>>>(s->vel, tex(s, 1 - p), tex(s, 2), dt, -1.f, s->n, m);
  S2D_LAUNCHED();
  k_dye_correct<<<grd, blk, 0, s->stream>>>(s->vel, tex(s, p), tex(s, 2), tex(s, 1 - p), dt, s->dparams,
                                            s->dsplats, s->n, m);
  S2D_LAUNCHED();
  s->dye_parity = 1 - p;
  return S2D_OK;
}

extern "C" int s2d_encode_reduce(s2d_solver* s) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  if (!s->reduced_valid) {
    // velocity came from a stage hook: the reference's two-level reduction
    const int groups = 256;
    k_reduce_speed<<<groups, 256, 0, s->stream>>>(s->vel, s->partials, s->n * s->n);
    S2D_LAUNCHED();
    k_reduce_dt<<<1, 256, 0, s->stream>>>(s->partials, groups, dt_slot(s, s->slot ^ 1), s->dparams);
    S2D_LAUNCHED();
  }
  s->slot ^= 1;
  s->reduced_valid = false;
  return S2D_OK;
}

static int sync_step_counter(s2d_solver* s) {
  const uint32_t v = s->step_index;
  S2D_CUDA(upload(s, s->step_counter, &v, sizeof(v)));
  return S2D_OK;
}

// stepIndex <- device counter (then counter + 1), done by the next step's first column kernel
static int enqueue_relatch(s2d_solver* s) {
  s->latch_pending = true;
  return S2D_OK;
}

// A fused step reads state[phase] (as w0) and writes the other two ring buffers, the
// packs, the velocity, the dye and the other dt slot, so one such step may run alongside
// the outstanding spectra (which read state[phase] of the step before it); the step after
// it writes that buffer, and the unfused tensor-core steps use the ring differently.
static int diag_order_step(s2d_solver* s, int substeps) {
  if (!s->diag_outstanding) return S2D_OK;
  if (s->diag_age == 0 && substeps <= 1 && !tc_unfused(s)) return S2D_OK;
  return diag_order(s);
}

extern "C" int s2d_step(s2d_solver* s, int substeps, unsigned flags) {
  S2D_USE_NOORDER(s);
  if (substeps < 0) return fail(S2D_ERR_ARG, "substeps < 0");
  DeviceGuard guard(s->dev);
  if (int rc = diag_order_step(s, substeps)) return rc;
  InStep in_step(s);
  if (!s->primed)
    if (int rc = s2d_encode_prime(s)) return rc;
  if (flags & S2D_STEP_RELATCH)
    if (int rc = sync_step_counter(s)) return rc;
  for (int i = 0; i < substeps; ++i) {
    if (flags & S2D_STEP_RELATCH)
      if (int rc = enqueue_relatch(s)) return rc;
    if (int rc = s2d_encode_step(s)) return rc;
    if (flags & S2D_STEP_DYE)
      if (int rc = s2d_encode_dye(s)) return rc;
    if (flags & S2D_STEP_REDUCE)
      if (int rc = s2d_encode_reduce(s)) return rc;
    ++s->diag_age;
  }
  return S2D_OK;
}

extern "C" int s2d_step_graph(s2d_solver* s, int substeps, unsigned flags) {
  S2D_USE_NOORDER(s);
  if (substeps < 0) return fail(S2D_ERR_ARG, "substeps < 0");
  DeviceGuard guard(s->dev);
  if (int rc = diag_order_step(s, substeps)) return rc;
  InStep in_step(s);
  if (!s->primed)
    if (int rc = s2d_encode_prime(s)) return rc;
  if (!s->packs_valid && !tc_unfused(s))
    if (int rc = enqueue_pack_prime(s)) return rc;
  if (flags & S2D_STEP_RELATCH)
    if (int rc = sync_step_counter(s)) return rc;
  for (int i = 0; i < substeps; ++i) {
    const GraphKey key{s->phase, s->slot, s->dye_parity, flags, s->hs.count > 0 ? 1 : 0, s->profiling ? 1 : 0};
    auto it = s->graphs.find(key);
    if (it == s->graphs.end()) {
      // capture one substep from the current host state, then restore it
      const int phase = s->phase, slot = s->slot, parity = s->dye_parity;
      const uint32_t si = s->step_index;
      const bool rv = s->reduced_valid;
      cudaGraph_t g = nullptr;
      cudaGraphExec_t ge = nullptr;
      const size_t ev_before = s->prof_events.size();
      S2D_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
      int rc = (flags & S2D_STEP_RELATCH) ? enqueue_relatch(s) : S2D_OK;
      if (!rc) rc = s2d_encode_step(s);
      if (!rc && (flags & S2D_STEP_DYE)) rc = s2d_encode_dye(s);
      if (!rc && (flags & S2D_STEP_REDUCE)) rc = s2d_encode_reduce(s);
      cudaError_t e = cudaStreamEndCapture(s->stream, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return fail(S2D_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&ge, g, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(S2D_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
      }
      s->phase = phase;
      s->slot = slot;
      s->dye_parity = parity;
      s->step_index = si;
      s->reduced_valid = rv;
      GraphEntry entry;
      entry.graph = g;
      entry.exec = ge;
      // event pairs recorded during capture belong to the graph's event nodes
      entry.events.assign(s->prof_events.begin() + ev_before, s->prof_events.end());
      s->prof_events.resize(ev_before);
      it = s->graphs.emplace(key, std::move(entry)).first;
    }
    S2D_CUDA(cudaGraphLaunch(it->second.exec, s->stream));
    if (!it->second.events.empty()) {
      // device times of this replay's kernels (the next replay re-records the events)
      S2D_CUDA(cudaStreamSynchronize(s->stream));
      for (auto& ev : it->second.events) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, std::get<1>(ev), std::get<2>(ev)) == cudaSuccess) {
          s->prof_ms[std::get<0>(ev)] += t;
          s->prof_cnt[std::get<0>(ev)] += 1;
        }
      }
    }
    // advance the host mirror exactly as the captured substep did
    s->phase = (s->phase + 1) % 3;
    s->step_index += 1;
    s->packs_valid = true;
    s->reduced_valid = true;
    if (flags & S2D_STEP_DYE) s->dye_parity ^= 1;
    if (flags & S2D_STEP_REDUCE) {
      s->slot ^= 1;
      s->reduced_valid = false;
    }
    ++s->diag_age;
  }
  return S2D_OK;
}

// ------------------------------------------------------------------ diagnostics
extern "C" int s2d_encode_diagnostics(s2d_solver* s) {
  S2D_USE(s);   // the previous spectra (and the copies before them) are done before this block is written
  DeviceGuard guard(s->dev);
  const int n = s->n;
  // fill the clear block; the spectra clear the other one for the next call
  const int b = s->diag_next;
  // the zonal mean reads the velocity, which the next step rewrites: on the main stream
  k_diag_zonal<<<diag_zonal_ctas(n), 256, 0, s->stream>>>(s->vel, diag_zonal(s, b), n);
  S2D_LAUNCHED();
  // the spectra of state[phase] on the diagnostics stream, alongside the next step (on the
  // main stream while a caller captures it into a graph of its own)
  const bool side = !stream_capturing(s->stream);
  if (side) {
    S2D_CUDA(cudaEventRecord(s->diag_ready, s->stream));
    S2D_CUDA(cudaStreamWaitEvent(s->diag_stream, s->diag_ready, 0));
  } else {
    // a captured graph may run any number of times: it clears the block it fills itself
    S2D_CUDA(cudaMemsetAsync(diag_fp64(s, b), 0, (sizeof(double) + sizeof(uint32_t)) * (size_t)(s->nbins + 2),
                             s->stream));
  }
  k_diag_tiles<<<diag_tiles(n), 256, diag_all_smem(n), side ? s->diag_stream : s->stream>>>(
      s->state[s->phase], diag_fp64(s, b), diag_u32(s, b), n, diag_fp64(s, 1 - b), diag_u32(s, 1 - b));
  S2D_LAUNCHED();
  if (side) {
    S2D_CUDA(cudaEventRecord(s->diag_done, s->diag_stream));
    s->diag_outstanding = true;
    s->diag_age = 0;
  }
  s->diag_last = b;
  s->diag_next = 1 - b;
  return S2D_OK;
}

extern "C" int s2d_copy_diagnostics(s2d_solver* s) {
  S2D_USE_NOORDER(s);
  if (s->read_state != 0) return S2D_OK;    // solver.js:561-563
  DeviceGuard guard(s->dev);
  // on the diagnostics stream, behind the spectra and the main stream's work so far (on the
  // main stream while a caller captures it): the block last filled, and the [dt, speed]
  // slot current now
  const bool side = !stream_capturing(s->stream);
  if (side) {
    S2D_CUDA(cudaEventRecord(s->diag_ready, s->stream));
    S2D_CUDA(cudaStreamWaitEvent(s->diag_stream, s->diag_ready, 0));
  }
  const cudaStream_t st = side ? s->diag_stream : s->stream;
  const int b = s->diag_last;
  const size_t off = diag_block_offset(s->nbins, s->n, b);
  S2D_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(s->h_base) + off, reinterpret_cast<char*>(s->diag) + off,
                           diag_block_bytes(s->nbins, s->n), cudaMemcpyDeviceToHost, st));
  S2D_CUDA(cudaMemcpyAsync(s->h_dt, dt_slot(s, s->slot), 2 * sizeof(float), cudaMemcpyDeviceToHost, st));
  set_host_diag_block(s, b);
  S2D_CUDA(cudaEventRecord(s->diag_event, st));
  s->read_state = 1;
  return S2D_OK;
}

// host-only (no upload flush): the Node-API addon polls from a worker thread
extern "C" int s2d_poll_diagnostics(s2d_solver* s) {
  S2D_USE_HOST(s);
  if (s->read_state != 1) return 0;
  return cudaEventQuery(s->diag_event) == cudaSuccess ? 1 : 0;
}

extern "C" int s2d_read_diagnostics(s2d_solver* s, double* spectrum, float* zonal, double* energy,
                                    double* enstrophy, float* dt, float* max_speed) {
  S2D_USE_NOORDER(s);
  if (s->read_state != 1) return S2D_NO_DATA;
  DeviceGuard guard(s->dev);
  cudaError_t e = cudaEventSynchronize(s->diag_event);
  s->read_state = 0;
  if (e != cudaSuccess) return fail(S2D_ERR_CUDA, cudaGetErrorString(e));
  const int nb = s->nbins;
  if (spectrum) std::memcpy(spectrum, s->h_diag, sizeof(double) * nb);
  if (zonal) std::memcpy(zonal, s->h_zonal, sizeof(float) * s->n);
  if (energy) *energy = s->h_diag[nb];
  if (enstrophy) *enstrophy = s->h_diag[nb + 1];
  if (dt) *dt = s->h_dt[0];
  if (max_speed) *max_speed = s->h_dt[1];
  return S2D_OK;
}

extern "C" int s2d_read_diagnostics_fixed(s2d_solver* s, float* spectrum, float* energy, float* enstrophy) {
  S2D_USE_NOORDER(s);
  DeviceGuard guard(s->dev);
  S2D_CUDA(cudaEventSynchronize(s->diag_event));
  const int nb = s->nbins;
  if (spectrum)
    for (int i = 0; i < nb; ++i) spectrum[i] = (float)(s->h_fixed[i] / 1e8);
  if (energy) *energy = (float)(s->h_fixed[nb] / 1e6);
  if (enstrophy) *enstrophy = (float)(s->h_fixed[nb + 1] / 1e6);
  return S2D_OK;
}

// ------------------------------------------------------------------ seeding
static int zero_other_states(s2d_solver* s) {
  const size_t cbytes = (size_t)s->n * s->n * sizeof(float2);
  S2D_CUDA(cudaMemsetAsync(s->state[1], 0, cbytes, s->stream));
  S2D_CUDA(cudaMemsetAsync(s->state[2], 0, cbytes, s->stream));
  return S2D_OK;
}

extern "C" int s2d_seed(s2d_solver* s, double k0, double amplitude, uint32_t seed) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  const int n = s->n;
  const size_t cbytes = (size_t)n * n * sizeof(float2);
  if (amplitude > 0) {
    const int parts = seed_parts_count(n);
    k_fill_spectrum<<<parts, 256, 0, s->stream>>>(s->state[0], s->seed_parts, n, k0, hash1(seed));
    S2D_LAUNCHED();
    k_scale_spectrum<<<std::min(parts, 1024), 256, 0, s->stream>>>(s->state[0], s->seed_parts, parts, n,
                                                                    amplitude);
    S2D_LAUNCHED();
  } else {
    S2D_CUDA(cudaMemsetAsync(s->state[0], 0, cbytes, s->stream));
  }
  s->phase = 0;
  s->packs_valid = false;
  return zero_other_states(s);
}

extern "C" int s2d_seed_band(s2d_solver* s, float kmin, float kmax, float rms, uint32_t seed) {
  S2D_USE(s);
  if (!(rms >= 0.f) || !(kmax >= kmin)) return fail(S2D_ERR_ARG, "bad band or rms");
  DeviceGuard guard(s->dev);
  const int n = s->n, parts = seed_parts_count(n);
  k_band_seed<<<parts, 256, 0, s->stream>>>(s->state[0], s->seed_parts, n, kmin, kmax, seed);
  S2D_LAUNCHED();
  k_scale_spectrum<<<std::min(parts, 1024), 256, 0, s->stream>>>(s->state[0], s->seed_parts, parts, n, rms);
  S2D_LAUNCHED();
  s->phase = 0;
  s->packs_valid = false;
  return zero_other_states(s);
}

static int check_finite(const float* v, size_t count) {
  for (size_t i = 0; i < count; ++i)
    if (!std::isfinite(v[i])) return fail(S2D_ERR_NAN, "non-finite value at index " + std::to_string(i));
  return S2D_OK;
}

// physical field staged (as floats) in the velocity buffer -> packA = (field, 0) -> FFT ->
// dealias mask into state 0 (solver.js:361-382)
static float* seed_staging(s2d_solver* s) { return reinterpret_cast<float*>(s->vel); }
static int seed_from_staging(s2d_solver* s) {
  const int n = s->n;
  if (int rc = materialize_packs(s)) return rc;   // packA is the scratch line here
  k_real_to_complex<<<cells_grid(n), 256, 0, s->stream>>>(seed_staging(s), s->packA, n * n);
  S2D_LAUNCHED();
  if (int rc = enqueue_fft2(s, s->packA, -1)) return rc;
  k_seed_mask<<<cells_grid(n), 256, 0, s->stream>>>(s->packA, s->state[0], n);
  S2D_LAUNCHED();
  S2D_CUDA(cudaStreamSynchronize(s->stream));   // a host field must outlive its copy
  s->phase = 0;
  s->packs_valid = false;
  s->reduced_valid = false;
  return zero_other_states(s);
}

extern "C" int s2d_seed_physical(s2d_solver* s, const float* field) {
  S2D_USE(s);
  if (!field) return fail(S2D_ERR_ARG, "field is null");
  const int n = s->n;
  if (int rc = check_finite(field, (size_t)n * n)) return rc;
  DeviceGuard guard(s->dev);
  S2D_CUDA(cudaMemcpyAsync(seed_staging(s), field, sizeof(float) * n * n, cudaMemcpyHostToDevice, s->stream));
  return seed_from_staging(s);
}

static int scenario_check(int kind, double param) {
  if (kind < S2D_SCENARIO_SHEAR_LAYER || kind > S2D_SCENARIO_POLYGON) return fail(S2D_ERR_ARG, "unknown scenario");
  if (kind == S2D_SCENARIO_MERGER && !std::isfinite(param)) return fail(S2D_ERR_ARG, "mergerSep must be finite");
  if (kind == S2D_SCENARIO_POLYGON) {
    const double c = std::floor(param + 0.5);
    if (!(c >= 1.0 && c <= S2D_SCENARIO_MAX_BLOBS)) return fail(S2D_ERR_ARG, "polygonN out of range");
  }
  return S2D_OK;
}

extern "C" int s2d_scenario_field(s2d_solver* s, int kind, double param, float* field_out) {
  S2D_USE(s);
  if (!field_out) return fail(S2D_ERR_ARG, "output is null");
  if (int rc = scenario_check(kind, param)) return rc;
  DeviceGuard guard(s->dev);
  const int n = s->n;
  // built in the stage-hook rhs buffer; state, packs and velocity are not touched
  float* tmp = reinterpret_cast<float*>(s->rhs);
  k_scenario<<<cells_grid(n), 256, 0, s->stream>>>(tmp, n, kind, param);
  S2D_LAUNCHED();
  S2D_CUDA(cudaMemcpyAsync(field_out, tmp, sizeof(float) * n * n, cudaMemcpyDeviceToHost, s->stream));
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  return S2D_OK;
}

extern "C" int s2d_paint_dye(s2d_solver* s, int pattern) {
  S2D_USE(s);
  if (pattern == S2D_DYE_NONE) return S2D_OK;
  if (pattern != S2D_DYE_BANDS) return fail(S2D_ERR_ARG, "unknown dye pattern");
  DeviceGuard guard(s->dev);
  const int m = s->m;
  k_paint_bands<<<(unsigned)(((size_t)m * m + 255) / 256), 256, 0, s->stream>>>(s->dye[s->dye_parity], m);
  S2D_LAUNCHED();
  return S2D_OK;
}

extern "C" int s2d_render(s2d_solver* s, int mode, float exposure, float vort_scale, float dye_gain, int width,
                          int height, void* rgba_out) {
  S2D_USE(s);
  if (!rgba_out) return fail(S2D_ERR_ARG, "output is null");
  if (mode < S2D_RENDER_DYE || mode > S2D_RENDER_SPEED) return fail(S2D_ERR_ARG, "unknown render mode");
  if (width <= 0 || height <= 0 || width > 16384 || height > 16384) return fail(S2D_ERR_ARG, "image size out of range");
  DeviceGuard guard(s->dev);
  const size_t px = (size_t)width * height;
  if (px > s->image_px) {
    if (s->image) cudaFree(s->image);
    s->image = nullptr;
    s->image_px = 0;
    S2D_CUDA(cudaMalloc(&s->image, px * sizeof(uchar4)));
    s->image_px = px;
  }
  // physical vorticity of the current state in the stage-hook rhs buffer
  const size_t cbytes = (size_t)s->n * s->n * sizeof(float2);
  S2D_CUDA(cudaMemcpyAsync(s->rhs, s->state[s->phase], cbytes, cudaMemcpyDeviceToDevice, s->stream));
  if (int rc = enqueue_fft2(s, s->rhs, +1)) return rc;
  const dim3 blk(16, 16), grd((width + 15) / 16, (height + 15) / 16);
  k_render<<<grd, blk, 0, s->stream>>>(s->image, width, height, s->rhs, s->vel, tex(s, s->dye_parity), s->n, s->m,
                                        mode, exposure, vort_scale, dye_gain);
  S2D_LAUNCHED();
  S2D_CUDA(cudaMemcpyAsync(rgba_out, s->image, px * sizeof(uchar4), cudaMemcpyDeviceToHost, s->stream));
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  return S2D_OK;
}

// ------------------------------------------------------------------ autotuner
static void drop_graphs(s2d_solver* s) {
  for (auto& kv : s->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    for (auto& ev : kv.second.events) {
      cudaEventDestroy(std::get<1>(ev));
      cudaEventDestroy(std::get<2>(ev));
    }
  }
  s->graphs.clear();
}

extern "C" int s2d_tune_variant_name(s2d_solver* s, int kind, int index, char* out, int cap) {
  S2D_USE(s);
  if (!out || cap <= 0) return fail(S2D_ERR_ARG, "output is null");
  const int count = kind == 0 ? s->ops->n_phys : kind == 1 ? spec_variants(s) : -1;
  if (count < 0) return fail(S2D_ERR_ARG, "kind is 0 (column) or 1 (row)");
  if (index < 0 || index >= count) return fail(S2D_ERR_ARG, "variant index out of range");
  const char* name = kind == 0 ? s->ops->phys[index].name
                     : index == s->ops->n_spec ? "tensor-core rows (split DFT-GEMM x-transforms)"
                                               : s->ops->spec[index].name;
  std::snprintf(out, (size_t)cap, "%s", name);
  return S2D_OK;
}

extern "C" int s2d_tune_select(s2d_solver* s, int phys, int spec) {
  S2D_USE(s);
  if (phys < 0 || phys >= s->ops->n_phys || spec < 0 || spec >= spec_variants(s))
    return fail(S2D_ERR_ARG, "variant index out of range");
  DeviceGuard guard(s->dev);
  s->phys_choice = phys;
  s->spec_choice = spec;
  drop_graphs(s);   // captured steps hold the previous shapes' kernels
  return S2D_OK;
}

extern "C" int s2d_autotune(s2d_solver* s, int steps, s2d_tune_report* report) {
  S2D_USE(s);
  if (steps < 1 || steps > 1000) return fail(S2D_ERR_ARG, "steps must be in 1..1000");
  DeviceGuard guard(s->dev);
  if (!s->primed)
    if (int rc = s2d_encode_prime(s)) return rc;
  const size_t cbytes = (size_t)s->n * s->n * sizeof(float2);
  // everything a trial changes: the state ring, the velocity, the dt slots, host counters
  float2* saved = nullptr;
  S2D_CUDA(cudaMalloc(&saved, 4 * cbytes + 64));
  float* saved_dt = reinterpret_cast<float*>(saved + 4 * (cbytes / sizeof(float2)));
  auto cp = [&](void* dst, const void* src, size_t b) {
    return cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToDevice, s->stream);
  };
  cudaError_t ce = cudaSuccess;
  for (int i = 0; i < 3 && ce == cudaSuccess; ++i) ce = cp(saved + i * (cbytes / sizeof(float2)), s->state[i], cbytes);
  if (ce == cudaSuccess) ce = cp(saved + 3 * (cbytes / sizeof(float2)), s->vel, cbytes);
  if (ce == cudaSuccess) ce = cp(saved_dt, s->dtbuf, 4 * sizeof(float));
  const int phase = s->phase, slot = s->slot;
  const uint32_t step_index = s->step_index;
  const bool reduced_valid = s->reduced_valid;
  auto restore = [&]() -> cudaError_t {
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cp(s->state[i], saved + i * (cbytes / sizeof(float2)), cbytes);
    if (e == cudaSuccess) e = cp(s->vel, saved + 3 * (cbytes / sizeof(float2)), cbytes);
    if (e == cudaSuccess) e = cp(s->dtbuf, saved_dt, 4 * sizeof(float));
    s->phase = phase;
    s->slot = slot;
    s->step_index = step_index;
    s->reduced_valid = reduced_valid;
    s->packs_valid = false;   // the packs are re-primed from the restored state
    return e;
  };
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  const bool was_profiling = s->profiling;
  s->profiling = false;
  int rc = ce == cudaSuccess ? S2D_OK : fail(S2D_ERR_CUDA, std::string("autotune setup: ") + cudaGetErrorString(ce));
  // one trial: restore, two untimed steps, then `steps` timed steps (step + fused CFL)
  auto trial = [&](float* us) -> int {
    if (cudaError_t e = restore(); e != cudaSuccess) return fail(S2D_ERR_CUDA, cudaGetErrorString(e));
    for (int k = 0; k < 2 + steps; ++k) {
      if (k == 2 && cudaEventRecord(e0, s->stream) != cudaSuccess) return fail(S2D_ERR_CUDA, "event");
      if (int r = s2d_encode_step(s)) return r;
      if (int r = s2d_encode_reduce(s)) return r;
    }
    if (cudaEventRecord(e1, s->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
      return fail(S2D_ERR_CUDA, "event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    *us = 1e3f * ms / steps;
    return S2D_OK;
  };
  s2d_tune_report rep{};
  rep.phys_variants = s->ops->n_phys;
  rep.spec_variants = spec_variants(s);
  const int p0 = s->phys_choice, q0 = s->spec_choice;
  // the tensor-core column stage has one shape: only the row shapes are tuned there
  const bool tc = is_tc(s);
  int best_p = p0, best_q = q0;
  if (!rc) {
    float best = 1e30f;
    for (int i = 0; i < s->ops->n_phys && !rc; ++i) {
      if (tc && i != p0) { rep.phys_us[i] = 0.f; continue; }
      s->phys_choice = i;
      rc = trial(&rep.phys_us[i]);
      if (!rc && rep.phys_us[i] < best) { best = rep.phys_us[i]; best_p = i; }
    }
    s->phys_choice = best_p;
    best = 1e30f;
    for (int j = 0; j < spec_variants(s) && !rc; ++j) {
      s->spec_choice = j;
      rc = trial(&rep.spec_us[j]);
      if (!rc && rep.spec_us[j] < best) { best = rep.spec_us[j]; best_q = j; }
    }
  }
  s->phys_choice = rc ? p0 : best_p;
  s->spec_choice = rc ? q0 : best_q;
  const cudaError_t re = restore();
  cudaStreamSynchronize(s->stream);
  cudaFree(saved);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  s->profiling = was_profiling;
  drop_graphs(s);
  if (rc) return rc;
  if (re != cudaSuccess) return fail(S2D_ERR_CUDA, std::string("autotune restore: ") + cudaGetErrorString(re));
  remember_choice(s);
  rep.phys_choice = s->phys_choice;
  rep.spec_choice = s->spec_choice;
  if (report) *report = rep;
  return S2D_OK;
}

// the part of reset() after the state is seeded (solver.js:429-443)
static int reset_after_seed(s2d_solver* s, int dye_pattern);

extern "C" int s2d_reset(s2d_solver* s, const float* field, double k0, double amplitude, uint32_t seed,
                         int dye_pattern) {
  S2D_USE(s);
  if (dye_pattern != S2D_DYE_NONE && dye_pattern != S2D_DYE_BANDS) return fail(S2D_ERR_ARG, "unknown dye pattern");
  DeviceGuard guard(s->dev);
  s->step_index = 0;
  s->sim_time = 0.0;
  s->dye_parity = 0;
  int rc = field ? s2d_seed_physical(s, field) : s2d_seed(s, k0, amplitude, seed);
  if (rc) return rc;
  return reset_after_seed(s, dye_pattern);
}

extern "C" int s2d_reset_scenario(s2d_solver* s, int kind, double param, int dye_pattern) {
  S2D_USE(s);
  if (dye_pattern != S2D_DYE_NONE && dye_pattern != S2D_DYE_BANDS) return fail(S2D_ERR_ARG, "unknown dye pattern");
  if (int rc = scenario_check(kind, param)) return rc;
  DeviceGuard guard(s->dev);
  s->step_index = 0;
  s->sim_time = 0.0;
  s->dye_parity = 0;
  k_scenario<<<cells_grid(s->n), 256, 0, s->stream>>>(seed_staging(s), s->n, kind, param);
  S2D_LAUNCHED();
  if (int rc = seed_from_staging(s)) return rc;
  return reset_after_seed(s, dye_pattern);
}

static int reset_after_seed(s2d_solver* s, int dye_pattern) {
  int rc;
  const size_t dbytes = (size_t)s->m * s->m * sizeof(ushort4);
  for (int i = 0; i < 3; ++i) S2D_CUDA(cudaMemsetAsync(s->dye[i], 0, dbytes, s->stream));
  if ((rc = s2d_paint_dye(s, dye_pattern))) return rc;
  const float dt0[2] = {s->configured ? s->hp.dt_max : 0.01f, 0.f};
  S2D_CUDA(cudaMemcpyAsync(dt_slot(s, s->slot), dt0, sizeof(dt0), cudaMemcpyHostToDevice, s->stream));
  S2D_CUDA(cudaMemsetAsync(s->force, 0, (size_t)s->n * s->n * sizeof(float2), s->stream));
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  s->primed = false;
  s->packs_valid = false;
  s->reduced_valid = false;
  return S2D_OK;
}

// ------------------------------------------------------------------ stage hooks
static int buffer_for(s2d_solver* s, int id, void** ptr, size_t* bytes) {
  const size_t cbytes = (size_t)s->n * s->n * sizeof(float2);
  switch (id) {
    case S2D_BUF_STATE0: case S2D_BUF_STATE1: case S2D_BUF_STATE2: *ptr = s->state[id]; *bytes = cbytes; return 0;
    case S2D_BUF_PACKA: *ptr = s->packA; *bytes = cbytes; return 0;
    case S2D_BUF_PACKB: *ptr = s->packB; *bytes = cbytes; return 0;
    case S2D_BUF_PHYSZ: *ptr = s->physZ; *bytes = cbytes; return 0;
    case S2D_BUF_RHS: *ptr = s->rhs; *bytes = cbytes; return 0;
    case S2D_BUF_FORCE: *ptr = s->force; *bytes = cbytes; return 0;
    case S2D_BUF_VEL: *ptr = s->vel; *bytes = cbytes; return 0;
    case S2D_BUF_DT: *ptr = dt_slot(s, s->slot); *bytes = 2 * sizeof(float); return 0;
    default: return fail(S2D_ERR_ARG, "unknown buffer id " + std::to_string(id));
  }
}

extern "C" int s2d_get_buffer(s2d_solver* s, int id, void* host, size_t bytes) {
  S2D_USE(s);
  if (!host) return fail(S2D_ERR_ARG, "host is null");
  void* p = nullptr;
  size_t sz = 0;
  if (int rc = buffer_for(s, id, &p, &sz)) return rc;
  DeviceGuard guard(s->dev);
  if (id == S2D_BUF_PACKA || id == S2D_BUF_PACKB)
    if (int rc = materialize_packs(s)) return rc;
  if (id == S2D_BUF_DT) {
    if (bytes < sz) return fail(S2D_ERR_ARG, "host buffer too small");
    float tmp[4] = {0, 0, 0, 0};
    S2D_CUDA(cudaMemcpyAsync(tmp, p, sz, cudaMemcpyDeviceToHost, s->stream));
    S2D_CUDA(cudaStreamSynchronize(s->stream));
    std::memcpy(host, tmp, std::min(bytes, sizeof(tmp)));
    return S2D_OK;
  }
  if (bytes > sz) return fail(S2D_ERR_ARG, "requested more bytes than the buffer holds");
  S2D_CUDA(cudaMemcpyAsync(host, p, bytes, cudaMemcpyDeviceToHost, s->stream));
  return check_device_error(s);
}

extern "C" int s2d_set_buffer(s2d_solver* s, int id, const void* host, size_t bytes) {
  S2D_USE(s);
  if (!host) return fail(S2D_ERR_ARG, "host is null");
  void* p = nullptr;
  size_t sz = 0;
  if (int rc = buffer_for(s, id, &p, &sz)) return rc;
  if (id == S2D_BUF_DT) bytes = std::min(bytes, sz);
  if (bytes > sz) return fail(S2D_ERR_ARG, "more bytes than the buffer holds");
  if (int rc = check_finite(static_cast<const float*>(host), bytes / sizeof(float))) return rc;
  DeviceGuard guard(s->dev);
  if (id == S2D_BUF_PACKA || id == S2D_BUF_PACKB)
    if (int rc = materialize_packs(s)) return rc;
  S2D_CUDA(cudaMemcpyAsync(p, host, bytes, cudaMemcpyHostToDevice, s->stream));
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  if (id <= S2D_BUF_PACKB) s->packs_valid = false;
  if (id == S2D_BUF_VEL) s->reduced_valid = false;
  return S2D_OK;
}

extern "C" int s2d_fft2(s2d_solver* s, int id, int inverse) {
  S2D_USE(s);
  float2* buf = nullptr;
  switch (id) {   // the buffers Solver.build registers (solver.js:133-136)
    case S2D_BUF_PACKA: buf = s->packA; break;
    case S2D_BUF_PACKB: buf = s->packB; break;
    case S2D_BUF_PHYSZ: buf = s->physZ; break;
    case S2D_BUF_FORCE: buf = s->force; break;
    default: return fail(S2D_ERR_UNREGISTERED, "buffer " + std::to_string(id) + " was never registered with the FFT");
  }
  DeviceGuard guard(s->dev);
  if (id == S2D_BUF_PACKA || id == S2D_BUF_PACKB) {
    if (int rc = materialize_packs(s)) return rc;
    s->packs_valid = false;
  }
  return enqueue_fft2(s, buf, inverse ? +1 : -1);
}

extern "C" int s2d_velocity_pack(s2d_solver* s, int state_index) {
  S2D_USE(s);
  if (state_index < 0 || state_index > 2) return fail(S2D_ERR_ARG, "state index out of range");
  DeviceGuard guard(s->dev);
  if (int rc = materialize_packs(s)) return rc;
  k_velocity_pack<<<cells_grid(s->n), 256, 0, s->stream>>>(s->state[state_index], s->packA, s->packB, s->n);
  S2D_LAUNCHED();
  s->packs_valid = false;
  return S2D_OK;
}

extern "C" int s2d_nl_pack(s2d_solver* s) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  if (int rc = materialize_packs(s)) return rc;
  k_nl_pack<<<cells_grid(s->n), 256, 0, s->stream>>>(s->packA, s->packB, s->physZ, s->vel, s->n);
  S2D_LAUNCHED();
  s->reduced_valid = false;
  return S2D_OK;
}

extern "C" int s2d_assemble(s2d_solver* s) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  k_assemble<<<cells_grid(s->n), 256, 0, s->stream>>>(s->physZ, s->force, dt_slot(s, s->slot), s->dparams,
                                                      s->rhs, s->n);
  S2D_LAUNCHED();
  return S2D_OK;
}

extern "C" int s2d_rk3_stage(s2d_solver* s, int stage) {
  S2D_USE(s);
  if (stage < 0 || stage > 2) return fail(S2D_ERR_ARG, "stage out of range");
  DeviceGuard guard(s->dev);
  const int p = s->phase;
  float2* w0 = s->state[p];
  float2* wc = s->state[(p + stage) % 3];
  float2* wo = s->state[(p + (stage == 1 ? 2 : 1)) % 3];
  const float* dt = dt_slot(s, s->slot);
  const unsigned g = cells_grid(s->n);
  if (stage == 0) k_rk3<0><<<g, 256, 0, s->stream>>>(w0, wc, wo, s->rhs, dt, s->dparams, s->n);
  else if (stage == 1) k_rk3<1><<<g, 256, 0, s->stream>>>(w0, wc, wo, s->rhs, dt, s->dparams, s->n);
  else k_rk3<2><<<g, 256, 0, s->stream>>>(w0, wc, wo, s->rhs, dt, s->dparams, s->n);
  S2D_LAUNCHED();
  s->packs_valid = false;
  return S2D_OK;
}

extern "C" int s2d_get_dye(s2d_solver* s, uint16_t* out) {
  S2D_USE(s);
  if (!out) return fail(S2D_ERR_ARG, "out is null");
  DeviceGuard guard(s->dev);
  S2D_CUDA(cudaMemcpyAsync(out, s->dye[s->dye_parity], (size_t)s->m * s->m * sizeof(ushort4),
                           cudaMemcpyDeviceToHost, s->stream));
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  return S2D_OK;
}

extern "C" int s2d_set_dye(s2d_solver* s, const uint16_t* in) {
  S2D_USE(s);
  if (!in) return fail(S2D_ERR_ARG, "in is null");
  DeviceGuard guard(s->dev);
  S2D_CUDA(cudaMemcpyAsync(s->dye[s->dye_parity], in, (size_t)s->m * s->m * sizeof(ushort4),
                           cudaMemcpyHostToDevice, s->stream));
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  return S2D_OK;
}

// ------------------------------------------------------------------ instrumentation
extern "C" int s2d_profile(s2d_solver* s, int enable) {
  S2D_USE(s);
  s->profiling = enable != 0;
  return S2D_OK;
}

extern "C" int s2d_profile_read(s2d_solver* s, double* ms, int* launches) {
  S2D_USE(s);
  DeviceGuard guard(s->dev);
  S2D_CUDA(cudaStreamSynchronize(s->stream));
  double acc[S2D_PROF_CLASSES] = {0};
  int cnt[S2D_PROF_CLASSES] = {0};
  for (int i = 0; i < S2D_PROF_CLASSES; ++i) {
    acc[i] = s->prof_ms[i];
    cnt[i] = s->prof_cnt[i];
    s->prof_ms[i] = 0.0;
    s->prof_cnt[i] = 0;
  }
  for (auto& ev : s->prof_events) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, std::get<1>(ev), std::get<2>(ev)) == cudaSuccess) {
      acc[std::get<0>(ev)] += t;
      cnt[std::get<0>(ev)] += 1;
    }
    cudaEventDestroy(std::get<1>(ev));
    cudaEventDestroy(std::get<2>(ev));
  }
  s->prof_events.clear();
  for (int i = 0; i < S2D_PROF_CLASSES; ++i) {
    if (ms) ms[i] = acc[i];
    if (launches) launches[i] = cnt[i];
  }
  return S2D_OK;
}
