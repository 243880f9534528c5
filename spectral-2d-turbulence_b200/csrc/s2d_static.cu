// s2d_static.cu -- CFL time step over caller-owned device buffers, allocating nothing.
//
// s2d_cfl_dt_static computes what s2d_encode_reduce computes (the maximum of
// |u|+|v| over a velocity field and the CFL step from it, reduce.wgsl:22-63)
// for callers that cannot allocate device memory: applications that reserve
// all GPU memory up front for their own allocator, or whose frame loop may not
// call cudaMalloc/cudaFree because those calls can synchronize the device.  The
// caller passes the velocity field and the two-float result buffer; the only
// scratch is the partial-maximum array below, a static device array that every
// GPU loading this library holds until the process exits.
#include <cuda.h>   // CUcontext / CUresult types only; the functions come from cudaGetDriverEntryPoint
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/s2d.h"
#include "s2d_device.cuh"

namespace s2d {
const char* ens_set_error(const std::string& m);   // shared error text (s2d_last_error)
}

namespace {

constexpr int kCellsPerPartial = 4096;      // cells reduced by one CTA of the first level
constexpr int kStaticThreads = 256;

// one partial maximum per 4096 cells: 4096 entries cover n*n <= 4096*4096
static __device__ __align__(256) float g_cfl_partials[S2D_CFL_STATIC_MAX_PARTIALS];

// level 1: CTA b writes partials[b] = max |u|+|v| over its 4096 cells (every slot used
// by a call is written before it is read, so nothing needs clearing between calls)
__global__ void k_static_speed(const float2* __restrict__ vel, long long cells, float* partials) {
  const long long begin = (long long)blockIdx.x * kCellsPerPartial;
  long long end = begin + kCellsPerPartial;
  if (end > cells) end = cells;
  float m = 0.f;
  for (long long i = begin + threadIdx.x; i < end; i += kStaticThreads) {
    const float2 v = vel[i];
    m = fmaxf(m, fabsf(v.x) + fabsf(v.y));
  }
  __shared__ float red[kStaticThreads / 32];
  m = s2d::warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    float s = threadIdx.x < kStaticThreads / 32 ? red[threadIdx.x] : 0.f;
    s = s2d::warp_max(s);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
  }
}

// level 2: one CTA reduces the partials and writes [dt, max |u|+|v|]
__global__ void k_static_dt(const float* __restrict__ partials, int count, float cfl, float dx, float dt_min,
                            float dt_max, float* dt_out) {
  float m = 0.f;
  for (int i = threadIdx.x; i < count; i += kStaticThreads) m = fmaxf(m, partials[i]);
  __shared__ float red[kStaticThreads / 32];
  m = s2d::warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    float s = threadIdx.x < kStaticThreads / 32 ? red[threadIdx.x] : 0.f;
    s = s2d::warp_max(s);
    if (threadIdx.x == 0) {
      float dt = dt_max;
      if (s > 1e-8f) dt = fminf(dt_max, cfl * dx / s);
      dt_out[0] = fmaxf(dt, dt_min);
      dt_out[1] = s;
    }
  }
}

// Device address of the static scratch, looked up once per CUDA context.  The array
// lives in the module loaded into a context, so its address belongs to that context:
// after cudaDeviceReset (the primary context is destroyed and a new one created) or
// with another driver-API context current, the address cached for an earlier context
// would be a dead or foreign pointer.  The cache is therefore keyed on the unique
// context id of the driver (cuCtxGetId), reached through cudaGetDriverEntryPoint so
// the library does not link libcuda.
using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);

struct ScratchSlot {
  unsigned long long ctx_id;
  float* addr;
};
constexpr int kCacheSlots = 64;
std::mutex g_addr_mutex;
ScratchSlot g_slots[kCacheSlots];
int g_slots_used = 0, g_slot_next = 0;
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;

int resolve_driver_entry_points() {
  if (g_ctx_get_current && g_ctx_get_id) return S2D_OK;
  void* f1 = nullptr;
  void* f2 = nullptr;
  cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
  cudaError_t e1 = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1);
  cudaError_t e2 = cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2);
  if (e1 != cudaSuccess || e2 != cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
      q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
    s2d::ens_set_error("s2d_cfl_dt_static: the driver does not provide cuCtxGetCurrent/cuCtxGetId");
    return S2D_ERR_CUDA;
  }
  g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(f1);
  g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(f2);
  return S2D_OK;
}

int symbol_address(float** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_partials);
  if (e != cudaSuccess || !p) {
    s2d::ens_set_error(std::string("s2d_cfl_dt_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return S2D_ERR_CUDA;
  }
  *out = static_cast<float*>(p);
  return S2D_OK;
}

int scratch_for_current_context(float** out) {
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (int rc = resolve_driver_entry_points()) return rc;
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) {
    s2d::ens_set_error("s2d_cfl_dt_static: cuCtxGetCurrent failed");
    return S2D_ERR_CUDA;
  }
  if (!ctx) {
    // no context current yet on this thread: the runtime call creates the current
    // device's primary context and makes it current
    float* p = nullptr;
    if (int rc = symbol_address(&p)) return rc;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) {
      s2d::ens_set_error("s2d_cfl_dt_static: no CUDA context is current");
      return S2D_ERR_NO_DEVICE;
    }
  }
  unsigned long long id = 0;
  if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) {
    s2d::ens_set_error("s2d_cfl_dt_static: cuCtxGetId failed");
    return S2D_ERR_CUDA;
  }
  for (int i = 0; i < g_slots_used; ++i)
    if (g_slots[i].ctx_id == id) {
      *out = g_slots[i].addr;
      return S2D_OK;
    }
  float* p = nullptr;
  if (int rc = symbol_address(&p)) return rc;
  // a context not seen before: remember it (the oldest entry makes room when full)
  const int slot = g_slots_used < kCacheSlots ? g_slots_used++ : (g_slot_next++ % kCacheSlots);
  g_slots[slot] = {id, p};
  *out = p;
  return S2D_OK;
}

}  // namespace

extern "C" int s2d_cfl_dt_static(const void* vel, int n, float cfl, float dt_min, float dt_max, void* dt_out,
                                 void* stream) {
  if (!vel || !dt_out) {
    s2d::ens_set_error("s2d_cfl_dt_static: null device pointer");
    return S2D_ERR_ARG;
  }
  if (n < 1 || n > S2D_CFL_STATIC_MAX_N) {
    s2d::ens_set_error("s2d_cfl_dt_static: n = " + std::to_string(n) + " is outside 1.." +
                       std::to_string(S2D_CFL_STATIC_MAX_N) + ", the size the static scratch array holds");
    return S2D_ERR_ARG;
  }
  float* partials = nullptr;
  if (int rc = scratch_for_current_context(&partials)) return rc;
  const long long cells = (long long)n * n;
  const int parts = (int)((cells + kCellsPerPartial - 1) / kCellsPerPartial);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_static_speed<<<parts, kStaticThreads, 0, st>>>(static_cast<const float2*>(vel), cells, partials);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    const float dx = (float)(2.0 * 3.14159265358979323846 / n);   // Params.dx (solver.js:317)
    k_static_dt<<<1, kStaticThreads, 0, st>>>(partials, parts, cfl, dx, dt_min, dt_max,
                                              static_cast<float*>(dt_out));
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    s2d::ens_set_error(std::string("s2d_cfl_dt_static: launch: ") + cudaGetErrorString(e));
    return S2D_ERR_CUDA;
  }
  return S2D_OK;
}
