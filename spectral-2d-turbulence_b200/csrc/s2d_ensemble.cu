// s2d_ensemble.cu -- many independent simulations of uneven grid sizes per launch.
//
// Every pass of the fused RK3 stage (physical columns, spectral row pairs) is ONE
// persistent launch over a work list of (instance, tile) items that mixes grid
// sizes 64..1024; each CTA loops over items, dispatching on the instance's N to
// the same tile functions the single-instance kernels use.  All instances share
// pooled buffers (state ring, packs, product spectra) addressed by per-instance
// offsets, and carry their own viscosity, beta, drag, forcing and dt.  A whole
// RK3 step (6 launches) is captured into a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/s2d.h"
#include "s2d_band.cuh"
#include "s2d_kernels.cuh"

using namespace s2d;

namespace s2d {
const char* ens_set_error(const std::string& m);
}

namespace {

int efail(int st, const std::string& m) {
  s2d::ens_set_error(m);
  return st;
}

#define E_CUDA(call)                                                                 \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return efail(S2D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define E_LAUNCHED() E_CUDA(cudaGetLastError())

struct EnsInst {
  DevParams p;           // per-instance coefficients
  float dt;              // fixed step
  int n;
  int tiles_a, tiles_b;
  long long off;         // first cell in the pooled arrays
  long long roff;        // first row in the pooled row flags
  const float2* tw;      // twiddle table of this n
};

constexpr int kEnsAThreads = 256;
constexpr int kEnsBThreads = 128;

template <int N> constexpr bool ens_size_ok() {
  return Tune<N>::A_THREADS == kEnsAThreads && Tune<N>::B_THREADS == kEnsBThreads;
}
static_assert(ens_size_ok<64>() && ens_size_ok<128>() && ens_size_ok<256>() && ens_size_ok<512>() &&
                  ens_size_ok<1024>(),
              "ensemble kernels assume one block shape for every grid size");

constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t kEnsASmem =
    cmax(cmax(cmax(Tune<64>::A_SMEM, Tune<128>::A_SMEM), cmax(Tune<256>::A_SMEM, Tune<512>::A_SMEM)),
         Tune<1024>::A_SMEM);
// one layout for every size: exchange lines, then the tile barrier (the default shapes
// stage no rows)
static_assert(!Tune<64>::PREFETCH && !Tune<128>::PREFETCH && !Tune<256>::PREFETCH && !Tune<512>::PREFETCH &&
                  !Tune<1024>::PREFETCH,
              "ensemble row tiles use no staging");
constexpr size_t kEnsBBarOff =
    cmax(cmax(cmax(Tune<64>::B_SMEM, Tune<128>::B_SMEM), cmax(Tune<256>::B_SMEM, Tune<512>::B_SMEM)),
         Tune<1024>::B_SMEM);
constexpr size_t kEnsBSmem = kEnsBBarOff + 16;

struct Pools {
  float2* s[3];
  float2 *pa, *pb, *z;
  // per instance row ky: 0 = the last row pass left PA/PB row ky all zero and unwritten
  // (the column pass reads no such row); starts at "may be nonzero"
  int* row_nz;
};

// MINB: resident CTAs per SM the register allocation must allow (a tuned choice)
template <int MINB>
__global__ void __launch_bounds__(kEnsAThreads, MINB)
    k_ens_phys(const EnsInst* __restrict__ inst, const int2* __restrict__ items, int nitems, Pools pool) {
  extern __shared__ float2 smem[];
  for (int k = blockIdx.x; k < nitems; k += gridDim.x) {
    const int2 it = items[k];
    const EnsInst& I = inst[it.x];
    PhysArgs a{};
    a.pa = pool.pa + I.off;
    a.pb = pool.pb + I.off;
    a.z = pool.z + I.off;
    a.params = &I.p;
    a.tw = I.tw;
    a.row_nz = pool.row_nz + I.roff;
    switch (I.n) {
      case 64: phys_cols_tile<64, 1>(a, it.y, smem); break;
      case 128: phys_cols_tile<128, 1>(a, it.y, smem); break;
      case 256: phys_cols_tile<256, 1>(a, it.y, smem); break;
      case 512: phys_cols_tile<512, 1>(a, it.y, smem); break;
      default: phys_cols_tile<1024, 1>(a, it.y, smem); break;
    }
    __syncthreads();
  }
}

// MINB: resident CTAs per SM the register allocation must allow.  Over pooled state far
// larger than L2 the row pass waits on HBM, and more CTAs in flight hide more of it even
// with some registers spilled to L1 (256 x 256^2: 761 -> 831 ensemble-steps/s going from
// four CTAs at 128 registers to six at 80); s2d_ensemble_autotune picks per ensemble.
// PAIR: the two inverse transforms of the next packs run as one two-line transform
// (half the barrier-separated passes, twice the registers for them).
template <int N, bool PAIR> using EnsTune = Tune<N, 16, 0, 0, false, PAIR>;
template <int MODE, int MINB, bool PAIR = false>
__global__ void __launch_bounds__(kEnsBThreads, MINB)
    k_ens_spec(const EnsInst* __restrict__ inst, const int2* __restrict__ items, int nitems, Pools pool, int phase,
               int* err) {
  extern __shared__ __align__(16) float2 smem[];
  const int st = MODE < 0 ? 0 : MODE;
  uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(smem) + kEnsBBarOff);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  uint32_t parity = 0;
  for (int k = blockIdx.x; k < nitems; k += gridDim.x, parity ^= 1u) {
    const int2 it = items[k];
    const EnsInst& I = inst[it.x];
    SpecArgs a{};
    a.z = pool.z + I.off;
    a.w0 = pool.s[phase] + I.off;
    a.wcur = pool.s[(phase + st) % 3] + I.off;
    a.wout = pool.s[(phase + (st == 1 ? 2 : 1)) % 3] + I.off;
    a.pa = pool.pa + I.off;
    a.pb = pool.pb + I.off;
    a.dt = &I.dt;
    a.params = &I.p;
    a.tw = I.tw;
    a.stochastic = I.p.force_amp > 0.f ? 1 : 0;
    a.err = err;
    a.row_nz = pool.row_nz + I.roff;
    switch (I.n) {
      case 64: spec_rows_tile<64, MODE, false, EnsTune<64, PAIR>>(a, it.y, smem, bar, parity); break;
      case 128: spec_rows_tile<128, MODE, false, EnsTune<128, PAIR>>(a, it.y, smem, bar, parity); break;
      case 256: spec_rows_tile<256, MODE, false, EnsTune<256, PAIR>>(a, it.y, smem, bar, parity); break;
      case 512: spec_rows_tile<512, MODE, false, EnsTune<512, PAIR>>(a, it.y, smem, bar, parity); break;
      default: spec_rows_tile<1024, MODE, false, EnsTune<1024, PAIR>>(a, it.y, smem, bar, parity); break;
    }
    __syncthreads();
  }
}

// ---- launch-shape variants of the two persistent stage kernels (index 0 = default)
constexpr int kEnsPhysMinb[] = {2, 3};      // resident CTAs per SM of each shape
constexpr int kEnsSpecMinb[] = {6, 4, 5, 4};
constexpr bool kEnsSpecPair[] = {false, false, false, true};
constexpr int kEnsNPhys = 2, kEnsNSpec = 4;

template <int MINB> cudaError_t ens_phys_attrs() {
  return cudaFuncSetAttribute(k_ens_phys<MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEnsASmem);
}
template <int MINB, bool PAIR = false> cudaError_t ens_spec_attrs() {
  cudaError_t e = cudaFuncSetAttribute(k_ens_spec<-1, MINB, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEnsBSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ens_spec<0, MINB, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEnsBSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ens_spec<1, MINB, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEnsBSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ens_spec<2, MINB, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEnsBSmem);
  return e;
}
const void* ens_phys_fn(int v) {
  return v == 1 ? (const void*)k_ens_phys<3> : (const void*)k_ens_phys<2>;
}
const void* ens_spec_fn(int v) {
  return v == 1 ? (const void*)k_ens_spec<1, 4> : v == 2 ? (const void*)k_ens_spec<1, 5>
         : v == 3 ? (const void*)k_ens_spec<1, 4, true> : (const void*)k_ens_spec<1, 6>;
}
void ens_launch_phys(int v, int grid, cudaStream_t st, const EnsInst* inst, const int2* items, int nitems, Pools pool) {
  if (v == 1) k_ens_phys<3><<<grid, kEnsAThreads, kEnsASmem, st>>>(inst, items, nitems, pool);
  else k_ens_phys<2><<<grid, kEnsAThreads, kEnsASmem, st>>>(inst, items, nitems, pool);
}
template <int MODE>
void ens_launch_spec_m(int v, int grid, cudaStream_t st, const EnsInst* inst, const int2* items, int nitems, Pools pool,
                       int phase, int* err) {
  if (v == 1) k_ens_spec<MODE, 4><<<grid, kEnsBThreads, kEnsBSmem, st>>>(inst, items, nitems, pool, phase, err);
  else if (v == 2) k_ens_spec<MODE, 5><<<grid, kEnsBThreads, kEnsBSmem, st>>>(inst, items, nitems, pool, phase, err);
  else if (v == 3)
    k_ens_spec<MODE, 4, true><<<grid, kEnsBThreads, kEnsBSmem, st>>>(inst, items, nitems, pool, phase, err);
  else k_ens_spec<MODE, 6><<<grid, kEnsBThreads, kEnsBSmem, st>>>(inst, items, nitems, pool, phase, err);
}
void ens_launch_spec(int mode, int v, int grid, cudaStream_t st, const EnsInst* inst, const int2* items, int nitems,
                     Pools pool, int phase, int* err) {
  if (mode < 0) ens_launch_spec_m<-1>(v, grid, st, inst, items, nitems, pool, phase, err);
  else if (mode == 0) ens_launch_spec_m<0>(v, grid, st, inst, items, nitems, pool, phase, err);
  else if (mode == 1) ens_launch_spec_m<1>(v, grid, st, inst, items, nitems, pool, phase, err);
  else ens_launch_spec_m<2>(v, grid, st, inst, items, nitems, pool, phase, err);
}

__global__ void k_ens_twiddles(float2* tw, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  double s, c;
  sincospi(2.0 * (double)m / (double)n, &s, &c);
  tw[m] = make_float2((float)c, (float)(-s));
}

// band seed of every instance: grid.y = instance, grid.x covers its cells
__global__ void k_ens_band(const EnsInst* __restrict__ inst, float2* s0, double* sums, const uint32_t* seeds,
                           float kmin, float kmax) {
  const EnsInst& I = inst[blockIdx.y];
  const int n = I.n;
  double acc = 0.0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    const float2 v = band_cell(seeds[blockIdx.y], n, idx / n, idx & (n - 1), kmin, kmax);
    s0[I.off + idx] = v;
    acc += (double)v.x * v.x + (double)v.y * v.y;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) atomicAdd(&sums[blockIdx.y], acc);
}

__global__ void k_ens_scale(const EnsInst* __restrict__ inst, float2* s0, const double* sums, float rms) {
  const EnsInst& I = inst[blockIdx.y];
  const int n = I.n;
  const double cur = sqrt(sums[blockIdx.y]) / ((double)n * n);
  const double sc = cur > 0.0 ? rms / cur : 1.0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    const float2 v = s0[I.off + idx];
    s0[I.off + idx] = make_float2((float)(v.x * sc), (float)(v.y * sc));
  }
}

// FP64 energy / enstrophy per instance (spectral2d.py:92-96)
__global__ void k_ens_energy(const EnsInst* __restrict__ inst, const float2* __restrict__ w, double* out) {
  const EnsInst& I = inst[blockIdx.y];
  const int n = I.n;
  const double n4 = (double)n * n * (double)n * n;
  double e = 0.0, z = 0.0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    const int c = idx & (n - 1), r = idx / n;
    const int kx = c < n / 2 ? c : c - n, ky = r < n / 2 ? r : r - n;
    const double k2 = (double)kx * kx + (double)ky * ky;
    const float2 a = w[I.off + idx];
    const double q = 0.5 * ((double)a.x * a.x + (double)a.y * a.y) / n4;
    z += q;
    if (k2 > 0) e += q / k2;
  }
  e = warp_sum(e);
  z = warp_sum(z);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[2 * blockIdx.y], e);
    atomicAdd(&out[2 * blockIdx.y + 1], z);
  }
}

bool ens_n_ok(int n) { return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024; }

template <int N> void tiles_of(int& a, int& b) {
  a = Tune<N>::A_GRID;
  b = Tune<N>::B_GRID;
}

}  // namespace

struct s2d_ensemble {
  int dev = 0, count = 0;
  cudaStream_t stream = nullptr;
  std::vector<EnsInst> hinst;
  std::vector<uint32_t> seeds;
  EnsInst* dinst = nullptr;
  uint32_t* dseeds = nullptr;
  int2 *items_a = nullptr, *items_b = nullptr;
  int nitems_a = 0, nitems_b = 0;
  int grid_a[kEnsNPhys] = {}, grid_b[kEnsNSpec] = {};   // persistent grids per launch shape
  int pv = 0, sv = 0;                                   // launch shapes in use
  Pools pool{};
  float2* tw = nullptr;
  double* sums = nullptr;    // 2 * count
  int* err = nullptr;        // device error word (bounded waits that gave up)
  long long cells = 0;
  int phase = 0;
  bool packs_valid = false;
  std::map<int, std::pair<cudaGraph_t, cudaGraphExec_t>> graphs;   // by starting phase
};

static void ens_free(s2d_ensemble* e) {
  for (auto& kv : e->graphs) {
    if (kv.second.second) cudaGraphExecDestroy(kv.second.second);
    if (kv.second.first) cudaGraphDestroy(kv.second.first);
  }
  void* ptrs[] = {e->dinst, e->dseeds, e->items_a, e->items_b, e->pool.s[0], e->pool.s[1], e->pool.s[2],
                  e->pool.pa, e->pool.pb, e->pool.z, e->pool.row_nz, e->tw, e->sums, e->err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (e->stream) cudaStreamDestroy(e->stream);
}

#define E_USE(e) \
  if (!(e)) return efail(S2D_ERR_ARG, "null ensemble handle")

extern "C" int s2d_ensemble_create(const s2d_instance_desc* descs, int count, int device, s2d_ensemble** out) {
  if (!out || !descs || count <= 0) return efail(S2D_ERR_ARG, "bad ensemble arguments");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return efail(S2D_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return efail(S2D_ERR_ARG, "device index out of range");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10)
    return efail(S2D_ERR_NO_DEVICE, "this library is built for sm_100a (B200) only");
  for (int i = 0; i < count; ++i) {
    if (!ens_n_ok(descs[i].n)) return efail(S2D_ERR_UNSUPPORTED_N, "ensemble grid sizes must be 64..1024, powers of two");
    if (descs[i].hyper_p < 0 || descs[i].hyper_p > 16) return efail(S2D_ERR_ARG, "hyper_p out of range");
  }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  s2d_ensemble* e = new s2d_ensemble();
  e->dev = device;
  e->count = count;
  auto bail = [&](cudaError_t err, const char* what) {
    ens_free(e);
    delete e;
    cudaSetDevice(prev);
    return efail(S2D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
  };
  cudaError_t err;
#define TRY(call, what)              \
  if ((err = (call)) != cudaSuccess) \
    return bail(err, what);
  TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "stream");
  // twiddle tables, one per distinct n
  std::map<int, long long> tw_off;
  long long tw_len = 0;
  for (int i = 0; i < count; ++i)
    if (!tw_off.count(descs[i].n)) {
      tw_off[descs[i].n] = tw_len;
      tw_len += descs[i].n;
    }
  TRY(cudaMalloc(&e->tw, sizeof(float2) * tw_len), "twiddles");
  for (auto& kv : tw_off) {
    k_ens_twiddles<<<(kv.first + 255) / 256, 256, 0, e->stream>>>(e->tw + kv.second, kv.first);
    TRY(cudaGetLastError(), "twiddle kernel");
  }
  // instances and work lists (largest grids first for balance)
  e->hinst.resize(count);
  e->seeds.resize(count);
  long long off = 0, roff = 0;
  for (int i = 0; i < count; ++i) {
    const s2d_instance_desc& d = descs[i];
    EnsInst& I = e->hinst[i];
    std::memset(&I, 0, sizeof(I));
    const int n = d.n;
    I.n = n;
    I.p.beta = d.beta;
    I.p.mu = d.drag;
    I.p.nu_h = d.nu_h;
    I.p.hyper_p = d.hyper_p;
    I.p.force_amp = d.force_amp;
    I.p.force_k = d.force_k;
    I.p.force_width = d.force_width;
    I.p.step_index = 0;
    I.p.dx = (float)(2.0 * M_PI / n);
    I.p.kcut = (float)(n / 3.0);
    I.p.force_norm = (float)(0.01 * n * n);
    I.p.n = n;
    I.dt = d.dt;
    switch (n) {
      case 64: tiles_of<64>(I.tiles_a, I.tiles_b); break;
      case 128: tiles_of<128>(I.tiles_a, I.tiles_b); break;
      case 256: tiles_of<256>(I.tiles_a, I.tiles_b); break;
      case 512: tiles_of<512>(I.tiles_a, I.tiles_b); break;
      default: tiles_of<1024>(I.tiles_a, I.tiles_b); break;
    }
    I.off = off;
    I.roff = roff;
    I.tw = e->tw + tw_off[n];
    off += (long long)n * n;
    roff += n;
    e->seeds[i] = d.seed;
  }
  e->cells = off;
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return e->hinst[a].n > e->hinst[b].n; });
  std::vector<int2> ia, ib;
  for (int i : order) {
    for (int t = 0; t < e->hinst[i].tiles_a; ++t) ia.push_back(make_int2(i, t));
    for (int t = 0; t < e->hinst[i].tiles_b; ++t) ib.push_back(make_int2(i, t));
  }
  e->nitems_a = (int)ia.size();
  e->nitems_b = (int)ib.size();
  TRY(cudaMalloc(&e->dinst, sizeof(EnsInst) * count), "instances");
  TRY(cudaMalloc(&e->dseeds, sizeof(uint32_t) * count), "seeds");
  TRY(cudaMalloc(&e->items_a, sizeof(int2) * ia.size()), "items");
  TRY(cudaMalloc(&e->items_b, sizeof(int2) * ib.size()), "items");
  TRY(cudaMalloc(&e->sums, sizeof(double) * 2 * count), "sums");
  TRY(cudaMalloc(&e->err, sizeof(int)), "error word");
  TRY(cudaMemsetAsync(e->err, 0, sizeof(int), e->stream), "memset");
  const size_t cbytes = sizeof(float2) * (size_t)off;
  for (int i = 0; i < 3; ++i) TRY(cudaMalloc(&e->pool.s[i], cbytes), "state pool");
  TRY(cudaMalloc(&e->pool.pa, cbytes), "pack pool");
  TRY(cudaMalloc(&e->pool.pb, cbytes), "pack pool");
  TRY(cudaMalloc(&e->pool.z, cbytes), "product pool");
  TRY(cudaMalloc(&e->pool.row_nz, sizeof(int) * (size_t)roff), "row flags");
  TRY(cudaMemsetAsync(e->pool.row_nz, 1, sizeof(int) * (size_t)roff, e->stream), "memset");   // nonzero words
  for (int i = 0; i < 3; ++i) TRY(cudaMemsetAsync(e->pool.s[i], 0, cbytes, e->stream), "memset");
  TRY(cudaMemsetAsync(e->pool.z, 0, cbytes, e->stream), "memset");
  TRY(cudaMemcpyAsync(e->dinst, e->hinst.data(), sizeof(EnsInst) * count, cudaMemcpyHostToDevice, e->stream), "copy");
  TRY(cudaMemcpyAsync(e->dseeds, e->seeds.data(), sizeof(uint32_t) * count, cudaMemcpyHostToDevice, e->stream), "copy");
  TRY(cudaMemcpyAsync(e->items_a, ia.data(), sizeof(int2) * ia.size(), cudaMemcpyHostToDevice, e->stream), "copy");
  TRY(cudaMemcpyAsync(e->items_b, ib.data(), sizeof(int2) * ib.size(), cudaMemcpyHostToDevice, e->stream), "copy");
  TRY(ens_phys_attrs<2>(), "attr");
  TRY(ens_phys_attrs<3>(), "attr");
  TRY(ens_spec_attrs<4>(), "attr");
  TRY(ens_spec_attrs<5>(), "attr");
  TRY(ens_spec_attrs<6>(), "attr");
  TRY((ens_spec_attrs<4, true>()), "attr");
  for (int v = 0; v < kEnsNPhys; ++v) {
    int occ = 0;
    TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ens_phys_fn(v), kEnsAThreads, kEnsASmem), "occupancy");
    e->grid_a[v] = std::min(e->nitems_a, std::max(1, occ) * prop.multiProcessorCount);
  }
  for (int v = 0; v < kEnsNSpec; ++v) {
    int occ = 0;
    TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ens_spec_fn(v), kEnsBThreads, kEnsBSmem), "occupancy");
    e->grid_b[v] = std::min(e->nitems_b, std::max(1, occ) * prop.multiProcessorCount);
  }
  TRY(cudaStreamSynchronize(e->stream), "sync");
#undef TRY
  cudaSetDevice(prev);
  *out = e;
  return S2D_OK;
}

extern "C" int s2d_ensemble_destroy(s2d_ensemble* e) {
  E_USE(e);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(e->dev);
  cudaStreamSynchronize(e->stream);
  ens_free(e);
  delete e;
  cudaSetDevice(prev);
  return S2D_OK;
}

extern "C" int s2d_ensemble_get_stream(s2d_ensemble* e, void** stream) {
  E_USE(e);
  if (!stream) return efail(S2D_ERR_ARG, "out is null");
  *stream = (void*)e->stream;
  return S2D_OK;
}

static int ens_check_err(s2d_ensemble* e) {
  int h = 0;
  E_CUDA(cudaMemcpy(&h, e->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    cudaMemset(e->err, 0, sizeof(int));
    return efail(S2D_ERR_CUDA, "a device-side wait for staged rows timed out; results of that step are invalid");
  }
  return S2D_OK;
}

extern "C" int s2d_ensemble_synchronize(s2d_ensemble* e) {
  E_USE(e);
  E_CUDA(cudaStreamSynchronize(e->stream));
  return ens_check_err(e);
}

extern "C" int s2d_ensemble_seed_band(s2d_ensemble* e, float kmin, float kmax, float rms) {
  E_USE(e);
  if (!(kmax >= kmin) || !(rms >= 0.f)) return efail(S2D_ERR_ARG, "bad band");
  const dim3 g(64, e->count);
  E_CUDA(cudaMemsetAsync(e->sums, 0, sizeof(double) * 2 * e->count, e->stream));
  k_ens_band<<<g, 256, 0, e->stream>>>(e->dinst, e->pool.s[0], e->sums, e->dseeds, kmin, kmax);
  E_LAUNCHED();
  k_ens_scale<<<g, 256, 0, e->stream>>>(e->dinst, e->pool.s[0], e->sums, rms);
  E_LAUNCHED();
  const size_t cbytes = sizeof(float2) * (size_t)e->cells;
  E_CUDA(cudaMemsetAsync(e->pool.s[1], 0, cbytes, e->stream));
  E_CUDA(cudaMemsetAsync(e->pool.s[2], 0, cbytes, e->stream));
  e->phase = 0;
  e->packs_valid = false;
  return S2D_OK;
}

extern "C" int s2d_ensemble_set_state(s2d_ensemble* e, int index, const float* spectrum) {
  E_USE(e);
  if (index < 0 || index >= e->count || !spectrum) return efail(S2D_ERR_ARG, "bad instance index");
  const EnsInst& I = e->hinst[index];
  const size_t bytes = sizeof(float2) * (size_t)I.n * I.n;
  for (size_t i = 0; i < bytes / sizeof(float); ++i)
    if (!std::isfinite(spectrum[i])) return efail(S2D_ERR_NAN, "non-finite value in spectrum");
  E_CUDA(cudaMemcpyAsync(e->pool.s[e->phase] + I.off, spectrum, bytes, cudaMemcpyHostToDevice, e->stream));
  E_CUDA(cudaStreamSynchronize(e->stream));
  e->packs_valid = false;
  return S2D_OK;
}

extern "C" int s2d_ensemble_get_state(s2d_ensemble* e, int index, float* spectrum) {
  E_USE(e);
  if (index < 0 || index >= e->count || !spectrum) return efail(S2D_ERR_ARG, "bad instance index");
  const EnsInst& I = e->hinst[index];
  E_CUDA(cudaMemcpyAsync(spectrum, e->pool.s[e->phase] + I.off, sizeof(float2) * (size_t)I.n * I.n,
                         cudaMemcpyDeviceToHost, e->stream));
  E_CUDA(cudaStreamSynchronize(e->stream));
  return ens_check_err(e);
}

static int ens_enqueue_step(s2d_ensemble* e) {
  const int p = e->phase;
  for (int st = 0; st < 3; ++st) {
    ens_launch_phys(e->pv, e->grid_a[e->pv], e->stream, e->dinst, e->items_a, e->nitems_a, e->pool);
    E_LAUNCHED();
    ens_launch_spec(st, e->sv, e->grid_b[e->sv], e->stream, e->dinst, e->items_b, e->nitems_b, e->pool, p, e->err);
    E_LAUNCHED();
  }
  e->phase = (p + 1) % 3;
  return S2D_OK;
}

extern "C" int s2d_ensemble_step(s2d_ensemble* e, int steps, int use_graph) {
  E_USE(e);
  if (steps < 0) return efail(S2D_ERR_ARG, "steps < 0");
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != e->dev) cudaSetDevice(e->dev);
  int rc = S2D_OK;
  if (!e->packs_valid) {
    ens_launch_spec(-1, e->sv, e->grid_b[e->sv], e->stream, e->dinst, e->items_b, e->nitems_b, e->pool, e->phase,
                    e->err);
    if (cudaGetLastError() != cudaSuccess) rc = efail(S2D_ERR_CUDA, "prime launch failed");
    e->packs_valid = true;
  }
  int done = 0;
  if (!rc && use_graph) {
    while (!rc && steps - done >= 3) {
      auto it = e->graphs.find(e->phase);
      if (it == e->graphs.end()) {
        const int p0 = e->phase;
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        cudaError_t err = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
        if (err != cudaSuccess) { rc = efail(S2D_ERR_CUDA, cudaGetErrorString(err)); break; }
        int r = S2D_OK;
        for (int i = 0; i < 3 && !r; ++i) r = ens_enqueue_step(e);
        err = cudaStreamEndCapture(e->stream, &g);
        e->phase = p0;
        if (r || err != cudaSuccess) {
          if (g) cudaGraphDestroy(g);
          rc = r ? r : efail(S2D_ERR_CUDA, cudaGetErrorString(err));
          break;
        }
        err = cudaGraphInstantiate(&ge, g, 0);
        if (err != cudaSuccess) {
          cudaGraphDestroy(g);
          rc = efail(S2D_ERR_CUDA, cudaGetErrorString(err));
          break;
        }
        it = e->graphs.emplace(p0, std::make_pair(g, ge)).first;
      }
      cudaError_t err = cudaGraphLaunch(it->second.second, e->stream);
      if (err != cudaSuccess) { rc = efail(S2D_ERR_CUDA, cudaGetErrorString(err)); break; }
      done += 3;   // three steps return the ring to the same phase
    }
  }
  for (; !rc && done < steps; ++done) rc = ens_enqueue_step(e);
  if (prev != e->dev) cudaSetDevice(prev);
  return rc;
}

extern "C" int s2d_ensemble_tune_variant_name(s2d_ensemble* e, int kind, int index, char* out, int cap) {
  E_USE(e);
  if (!out || cap <= 0) return efail(S2D_ERR_ARG, "output is null");
  const int count = kind == 0 ? kEnsNPhys : kind == 1 ? kEnsNSpec : -1;
  if (count < 0 || index < 0 || index >= count) return efail(S2D_ERR_ARG, "variant out of range");
  std::snprintf(out, (size_t)cap, "%d CTAs/SM%s", kind == 0 ? kEnsPhysMinb[index] : kEnsSpecMinb[index],
                kind == 1 && kEnsSpecPair[index] ? ", paired inverse transforms" : "");
  return S2D_OK;
}

extern "C" int s2d_ensemble_autotune(s2d_ensemble* e, int steps, s2d_tune_report* report) {
  E_USE(e);
  if (steps < 1 || steps > 300) return efail(S2D_ERR_ARG, "steps must be in 1..300");
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != e->dev) cudaSetDevice(e->dev);
  const size_t cbytes = sizeof(float2) * (size_t)e->cells;
  float2* saved = nullptr;
  int rc = S2D_OK;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaMalloc(&saved, 3 * cbytes) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess)
    rc = efail(S2D_ERR_CUDA, "autotune: out of device memory for the saved state");
  const int phase = e->phase;
  auto restore = [&]() {
    for (int i = 0; i < 3; ++i)
      cudaMemcpyAsync(e->pool.s[i], saved + i * e->cells, cbytes, cudaMemcpyDeviceToDevice, e->stream);
    e->phase = phase;
    e->packs_valid = false;
  };
  if (!rc)
    for (int i = 0; i < 3; ++i)
      cudaMemcpyAsync(saved + i * e->cells, e->pool.s[i], cbytes, cudaMemcpyDeviceToDevice, e->stream);
  auto trial = [&](float* us) -> int {
    restore();
    if (int r = s2d_ensemble_step(e, 1, 0)) return r;   // primes, one untimed step
    cudaEventRecord(e0, e->stream);
    if (int r = s2d_ensemble_step(e, steps, 0)) return r;
    cudaEventRecord(e1, e->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) return efail(S2D_ERR_CUDA, "autotune: event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    *us = 1e3f * ms / steps;
    return S2D_OK;
  };
  s2d_tune_report rep{};
  rep.phys_variants = kEnsNPhys;
  rep.spec_variants = kEnsNSpec;
  const int pv0 = e->pv, sv0 = e->sv;
  int best_p = pv0, best_s = sv0;
  if (!rc) {
    float best = 1e30f;
    for (int v = 0; v < kEnsNPhys && !rc; ++v) {
      e->pv = v;
      rc = trial(&rep.phys_us[v]);
      if (!rc && rep.phys_us[v] < best) { best = rep.phys_us[v]; best_p = v; }
    }
    e->pv = best_p;
    best = 1e30f;
    for (int v = 0; v < kEnsNSpec && !rc; ++v) {
      e->sv = v;
      rc = trial(&rep.spec_us[v]);
      if (!rc && rep.spec_us[v] < best) { best = rep.spec_us[v]; best_s = v; }
    }
  }
  e->pv = rc ? pv0 : best_p;
  e->sv = rc ? sv0 : best_s;
  if (saved) restore();
  cudaStreamSynchronize(e->stream);
  if (saved) cudaFree(saved);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  for (auto& kv : e->graphs) {          // captured with the previous shapes
    if (kv.second.second) cudaGraphExecDestroy(kv.second.second);
    if (kv.second.first) cudaGraphDestroy(kv.second.first);
  }
  e->graphs.clear();
  if (prev != e->dev) cudaSetDevice(prev);
  if (rc) return rc;
  rep.phys_choice = e->pv;
  rep.spec_choice = e->sv;
  if (report) *report = rep;
  return S2D_OK;
}

extern "C" int s2d_ensemble_tune_select(s2d_ensemble* e, int phys, int spec) {
  E_USE(e);
  if (phys < 0 || phys >= kEnsNPhys || spec < 0 || spec >= kEnsNSpec)
    return efail(S2D_ERR_ARG, "ensemble shape index out of range");
  e->pv = phys;
  e->sv = spec;
  for (auto& kv : e->graphs) {          // captured with the previous shapes
    if (kv.second.second) cudaGraphExecDestroy(kv.second.second);
    if (kv.second.first) cudaGraphDestroy(kv.second.first);
  }
  e->graphs.clear();
  return S2D_OK;
}

extern "C" int s2d_ensemble_energy(s2d_ensemble* e, double* energy, double* enstrophy) {
  E_USE(e);
  E_CUDA(cudaMemsetAsync(e->sums, 0, sizeof(double) * 2 * e->count, e->stream));
  const dim3 g(64, e->count);
  k_ens_energy<<<g, 256, 0, e->stream>>>(e->dinst, e->pool.s[e->phase], e->sums);
  E_LAUNCHED();
  std::vector<double> h(2 * e->count);
  E_CUDA(cudaMemcpyAsync(h.data(), e->sums, sizeof(double) * 2 * e->count, cudaMemcpyDeviceToHost, e->stream));
  E_CUDA(cudaStreamSynchronize(e->stream));
  for (int i = 0; i < e->count; ++i) {
    if (energy) energy[i] = h[2 * i];
    if (enstrophy) enstrophy[i] = h[2 * i + 1];
  }
  return S2D_OK;
}
