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

// device address of the static scratch, looked up once per device
constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
float* g_addr[kMaxDevices] = {nullptr};

int scratch_for_current_device(float** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    s2d::ens_set_error(std::string("s2d_cfl_dt_static: cudaGetDevice: ") + cudaGetErrorString(e));
    return S2D_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    s2d::ens_set_error("s2d_cfl_dt_static: device ordinal out of range");
    return S2D_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_cfl_partials);
    if (e != cudaSuccess || !p) {
      s2d::ens_set_error(std::string("s2d_cfl_dt_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return S2D_ERR_CUDA;
    }
    g_addr[dev] = static_cast<float*>(p);
  }
  *out = g_addr[dev];
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
  if (int rc = scratch_for_current_device(&partials)) return rc;
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
