// s2d_aux_kernels.cuh -- forcing, CFL reduction, diagnostics, seeding, dye, tables.
#pragma once
#include <cuda_fp16.h>
#include "s2d_band.cuh"
#include "s2d_device.cuh"
#include "s2d_dye.cuh"

namespace s2d {

// ------------------------------------------------------------------ tables (FP64 generation)
// exp(-2 pi i m / n) for m < n, generated in FP64 and rounded once to float.
__global__ void k_twiddles(float2* tw, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  double s, c;
  sincospi(2.0 * (double)m / (double)n, &s, &c);
  tw[m] = make_float2((float)c, (float)(-s));
}

// digit reversal over the reversed radix list [4,..,4,(2)] (fft.wgsl:32-40, fft_ref.py:19-24)
__global__ void k_digit_reverse(uint32_t* out, int n, int stages, int has_r2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t v = (uint32_t)i, o = 0;
  if (has_r2) {
    o = o * 2u + (v % 2u);
    v /= 2u;
  }
  for (int s = 0; s < stages; ++s) {
    o = o * 4u + (v % 4u);
    v /= 4u;
  }
  out[i] = o;
}

__global__ void k_wavenumbers(float* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = wn_rt(i, n);
}

__global__ void k_mask_table(uint8_t* out, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  const float kcut = (float)(n / 3.0);
  const float kx = wn_rt(idx & (n - 1), n), ky = wn_rt(idx / n, n);
  out[idx] = (fabsf(kx) < kcut && fabsf(ky) < kcut) ? 1 : 0;
}

// ------------------------------------------------------------------ pointer forcing (force.wgsl:5-27)

__global__ void k_pointer_force(float2* force, const DevSplats* __restrict__ S, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  const float nf = (float)n;
  const float x = ((float)(idx & (n - 1)) + 0.5f) / nf;
  const float y = ((float)(idx / n) + 0.5f) / nf;
  float total = 0.f;
  const int cnt = S->count;
  for (int i = 0; i < cnt; ++i) {
    const DevSplat s = S->items[i];
    const float rx = sepf(x, s.x), ry = sepf(y, s.y);
    const float r2 = rx * rx + ry * ry;
    const float sig2 = fmaxf(s.radius * s.radius, 1e-8f);
    if (r2 < 9.f * sig2) {
      const float g = expf(-r2 / sig2);
      total += 2.f * s.amp * g * (s.vx * ry - s.vy * rx) / sig2;
    }
  }
  force[idx] = make_float2(total, 0.f);
}

// ------------------------------------------------------------------ CFL reduction (reduce.wgsl:22-63)
__global__ void k_reduce_speed(const float2* __restrict__ vel, float* partials, int ncells) {
  float m = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncells; i += gridDim.x * blockDim.x) {
    const float2 v = vel[i];
    m = fmaxf(m, fabsf(v.x) + fabsf(v.y));
  }
  __shared__ float red[32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    float s = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
    s = warp_max(s);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
  }
}

__global__ void k_reduce_dt(const float* __restrict__ partials, int count, float* dt_out,
                            const DevParams* __restrict__ params) {
  float m = 0.f;
  for (int i = threadIdx.x; i < count; i += blockDim.x) m = fmaxf(m, partials[i]);
  __shared__ float red[32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    float s = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
    s = warp_max(s);
    if (threadIdx.x == 0) {
      dt_out[0] = cfl_dt(*params, s);
      dt_out[1] = s;
    }
  }
}

// ------------------------------------------------------------------ seeding
// seed.wgsl:4-17: dst = src * mask, k = 0 cleared
__global__ void k_seed_mask(const float2* __restrict__ src, float2* dst, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  const float kcut = (float)(n / 3.0);
  const float kx = wn_rt(idx & (n - 1), n), ky = wn_rt(idx / n, n);
  if (kx == 0.f && ky == 0.f) {
    dst[idx] = make_float2(0.f, 0.f);
    return;
  }
  dst[idx] = (fabsf(kx) < kcut && fabsf(ky) < kcut) ? src[idx] : make_float2(0.f, 0.f);
}

// real field -> complex (value, 0) (solver.js:363-367)
// zero the rows of the packs that the row kernel flagged as all zero and left unwritten
__global__ void k_zero_flagged_rows(float2* pa, float2* pb, const int* __restrict__ row_nz, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  if (row_nz[idx / n] == 0) {
    pa[idx] = make_float2(0.f, 0.f);
    pb[idx] = make_float2(0.f, 0.f);
  }
}

__global__ void k_real_to_complex(const float* __restrict__ src, float2* dst, int ncells) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ncells) dst[i] = make_float2(src[i], 0.f);
}

// fillSpectrum (solver.js:384-418) in double precision like the JS host code:
// unscaled Float32 values plus per-CTA partial sums of amp^2.
__global__ void k_fill_spectrum(float2* data, double* partial, int n, double k0, uint32_t salt) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (idx < n * n) {
    const int col = idx & (n - 1), row = idx / n;
    const double kcut = n / 3.0;
    const int kxi = col < n / 2 ? col : col - n;
    const int kyi = row < n / 2 ? row : row - n;
    float2 val = make_float2(0.f, 0.f);
    if (!((kxi == 0 && kyi == 0) || abs(kxi) >= kcut || abs(kyi) >= kcut)) {
      const double kr = hypot((double)kxi, (double)kyi);
      const double q = kr / k0;
      const double q2 = q * q, q4 = q2 * q2;
      const double env = kr * kr / (1.0 + q4 * q4);
      const double amp = sqrt(env);
      const bool canon = kyi > 0 || (kyi == 0 && kxi > 0);
      const int hr = canon ? row : (n - row) % n;
      const int hc = canon ? col : (n - col) % n;
      const double sgn = canon ? 1.0 : -1.0;
      const double phase = 2.0 * 3.14159265358979323846 * (double)hash1((uint32_t)(hr * n + hc) ^ salt) / 4294967296.0;
      double s, c;
      sincos(phase, &s, &c);
      val = make_float2((float)(amp * c), (float)(sgn * amp * s));
      acc = amp * amp;
    }
    data[idx] = val;
  }
  acc = warp_sum(acc);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

// band-limited Gaussian spectrum (s2d_band.cuh) with per-CTA partial sums of |w|^2
__global__ void k_band_seed(float2* data, double* partial, int n, float kmin, float kmax, uint32_t seed) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (idx < n * n) {
    const float2 v = band_cell(seed, n, idx / n, idx & (n - 1), kmin, kmax);
    data[idx] = v;
    acc = (double)v.x * v.x + (double)v.y * v.y;
  }
  acc = warp_sum(acc);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

// scale = amplitude / (sqrt(sum)/n^2); data *= scale (Float32Array *= double, solver.js:411-417)
__global__ void k_scale_spectrum(float2* data, const double* partial, int nparts, int n, double amplitude) {
  __shared__ double scale;
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int i = 0; i < nparts; ++i) sum += partial[i];
    const double rms = sqrt(sum) / ((double)n * (double)n);
    scale = rms > 0.0 ? amplitude / rms : 1.0;
  }
  __syncthreads();
  const double sc = scale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x) {
    const float2 v = data[i];
    data[i] = make_float2((float)((double)v.x * sc), (float)((double)v.y * sc));
  }
}

// ------------------------------------------------------------------ diagnostics
// The zonal mean of u (spectrum.wgsl:41-68), FP64 sums: one warp per row, a lane's loads
// issued sixteen at a time (a whole 1024-cell row in one round trip; with one load in
// flight per lane the zonal mean took 6.2 us alone at 1024^2).  Lane order i = lane + 32 j
// within a row, then the warp sum.
__host__ __device__ constexpr int diag_zonal_ctas(int n) { return (n + 7) / 8; }
__global__ void __launch_bounds__(256) k_diag_zonal(const float2* __restrict__ vel, float* zonal, int n) {
  constexpr int kBatch = 16;
  const int lane = threadIdx.x & 31;
  const int row = (int)blockIdx.x * 8 + (int)(threadIdx.x >> 5);
  if (row >= n) return;
  const int nq = n / 2;   // float4 (two velocity cells) per row
  const float4* r4 = reinterpret_cast<const float4*>(vel + (size_t)row * n);
  double acc = 0.0;
  for (int base = lane; base < nq; base += 32 * kBatch) {
    float4 t[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; ++j)
      t[j] = base + 32 * j < nq ? __ldcs(r4 + base + 32 * j) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int j = 0; j < kBatch; ++j)
      if (base + 32 * j < nq) {
        acc += (double)t[j].x;
        acc += (double)t[j].z;
      }
  }
  acc = warp_sum(acc);
  if (lane == 0) zonal[row] = (float)(acc / n);
}

// Both spectra in one pass over the state: the FP64 radial spectrum, energy and
// enstrophy (spectral2d.py:92-104) and the reference's u32 fixed-point bins,
// truncating, in the dealias band (spectrum.wgsl:19-39).
//
// A CTA takes a k-space tile of TW x TH cells (TW = min(64, n), TW * TH = 2048).  The
// cells of a tile span fewer than kDiagSpan radial bins (its diagonal is < 72), so each
// lane of a warp keeps its own FP64 window of kDiagSpan bins from the tile's lowest bin
// (FP64 shared-memory adds to one word serialise; with per-lane windows only the same
// lane of different warps can meet on a word).  A thread takes 8 consecutive cells of a row,
// whose bins change slowly along kx, and adds each run of equal bins once; a bin outside
// the window (none by construction) goes straight to global memory.  The windows are
// summed over the 32 lanes in a fixed order and each nonzero bin is added to global
// memory once per CTA (18.5 -> 14.4 us at 1024^2 against one shared FP64 array whose
// words the 8 threads of a tile row hit together).  The u32 fixed-point bins use one
// shared array: the u32 sums wrap
// mod 2^32 in any order, so the result equals per-cell atomics bit for bit.  The sums
// accumulate into a block that is zero on entry; the first CTA zeroes the caller's other
// block (clear_out, clear_bins), so calls that alternate between two blocks need no clear
// of their own.
//
// Per cell: the f32 bin round(sqrtf(k2)) is the reference's; the FP64 bin
// floor(sqrt(k2) + 0.5) is the same integer corrected by one step with integer tests
// (b^2 - b < k2 <= b^2 + b; sqrt(k2) is never a half-integer).  n^4 is a power of two,
// so scaling by its reciprocal is the division, bit for bit.
constexpr int kDiagCells = 8;
constexpr int kDiagSpan = 80;
constexpr int kDiagStride = kDiagSpan + 1;   // odd double stride: the 32 lanes' windows fall in distinct banks
__host__ __device__ constexpr int diag_tile_w(int n) { return n < 64 ? n : 64; }
__host__ __device__ constexpr int diag_tile_h(int n) { return 2048 / diag_tile_w(n) < n ? 2048 / diag_tile_w(n) : n; }
__host__ __device__ constexpr int diag_tiles(int n) { return (n / diag_tile_w(n)) * (n / diag_tile_h(n)); }
__host__ __device__ constexpr size_t diag_all_smem(int n) {
  return sizeof(double) * (32 * kDiagStride + 2) + sizeof(uint32_t) * (size_t)(n / 2 + 3);
}
// smallest |k| over a range of FFT indices [i0, i0 + len) (wrapped wavenumbers)
__device__ __forceinline__ int diag_min_abs_wn(int i0, int len, int n) {
  if (len >= n) return 0;
  const int a = i0 < n / 2 ? i0 : i0 - n, b = (i0 + len - 1) < n / 2 ? i0 + len - 1 : i0 + len - 1 - n;
  if (a <= 0 && b >= 0) return 0;
  if (a > b) return 0;   // the range crosses n/2 (both signs present)
  return min(abs(a), abs(b));
}
__global__ void __launch_bounds__(256) k_diag_tiles(const float2* __restrict__ w, double* out, uint32_t* bins,
                                                    int n, double* clear_out, uint32_t* clear_bins) {
  if (blockIdx.x == 0) {   // zero the other block's sums for the next launch
    for (int i = threadIdx.x; i < n / 2 + 3; i += blockDim.x) {
      clear_out[i] = 0.0;
      clear_bins[i] = 0u;
    }
  }
  const int tile = (int)blockIdx.x;
  extern __shared__ double win[];                      // [32 lanes][kDiagStride], then 2 totals
  double* const tot = win + 32 * kDiagStride;
  uint32_t* const fhist = reinterpret_cast<uint32_t*>(tot + 2);
  const int nb = n / 2 + 1;
  const int lane = threadIdx.x & 31;
  static_assert((32 * kDiagStride + 2) % 2 == 0, "windows and totals cleared in 16-byte stores");
  for (int i = threadIdx.x; i < (32 * kDiagStride + 2) / 2; i += blockDim.x)
    reinterpret_cast<double2*>(win)[i] = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < nb + 2; i += blockDim.x) fhist[i] = 0u;
  const int tw = diag_tile_w(n), th = diag_tile_h(n), per_row = tw / kDiagCells;
  const int tiles_x = n / tw;
  const int col0 = (tile % tiles_x) * tw, row0 = (tile / tiles_x) * th;
  // lowest bin of the tile, less one for rounding: floor(sqrt(min k2)) - 1, and at most
  // the last bin (|k| beyond n/2 is binned there)
  const int mkx = diag_min_abs_wn(col0, tw, n), mky = diag_min_abs_wn(row0, th, n);
  const int lo = min(max((int)floorf(sqrtf((float)(mkx * mkx + mky * mky))) - 1, 0), nb - 1);
  double* const my = win + lane * kDiagStride;
  __syncthreads();
  const double inv_n4 = 1.0 / ((double)n * n * (double)n * n);
  const float inv_n4f = 1.f / ((float)n * (float)n * ((float)n * (float)n));
  const float kcut = (float)(n / 3.0);
  double ene = 0.0, ens = 0.0;
  uint32_t fe = 0u, fz = 0u;
  if ((int)threadIdx.x < th * per_row) {
    const int row = row0 + (int)threadIdx.x / per_row;
    const int c0 = col0 + ((int)threadIdx.x % per_row) * kDiagCells;
    const int ky = row < n / 2 ? row : row - n;
    const float kyf = (float)ky;
    const float4* p = reinterpret_cast<const float4*>(w + (size_t)row * n + c0);
    float2 v[kDiagCells];
#pragma unroll
    for (int q = 0; q < kDiagCells / 2; ++q) {
      const float4 t = p[q];
      v[2 * q] = make_float2(t.x, t.y);
      v[2 * q + 1] = make_float2(t.z, t.w);
    }
    int cur_b = -1, cur_fb = -1;
    double cur_e = 0.0;
    uint32_t cur_f = 0u;
#pragma unroll
    for (int j = 0; j < kDiagCells; ++j) {
      const int col = c0 + j;
      const int kx = col < n / 2 ? col : col - n;
      const float2 a = v[j];
      const int k2i = kx * kx + ky * ky;
      const float kxf = (float)kx;
      const float k2f = kxf * kxf + kyf * kyf;                       // exact (k2 < 2^24)
      const int fb_raw = (int)(sqrtf(k2f) + 0.5f);
      // FP64
      const double z = 0.5 * ((double)a.x * a.x + (double)a.y * a.y) * inv_n4;
      ens += z;
      if (k2i > 0) {
        // z / k2 as z times the correctly rounded reciprocal: within 1.5 ulp of the
        // quotient, far inside the 1e-12 the FP64 diagnostics are held to
        const double e = z * __drcp_rn((double)k2i);
        ene += e;
        int b = fb_raw;
        if (b * b - b >= k2i) --b;
        else if (b * b + b < k2i) ++b;
        b = b < nb - 1 ? b : nb - 1;
        if (b != cur_b) {
          if (cur_b >= 0) {
            // this lane's window is shared only with the same lane of the other warps
            const unsigned r = (unsigned)(cur_b - lo);
            if (r < (unsigned)kDiagSpan) atomicAdd(my + r, cur_e);
            else atomicAdd(out + cur_b, cur_e);
          }
          cur_b = b;
          cur_e = 0.0;
        }
        cur_e += e;
      }
      // u32 fixed point
      if (k2f != 0.f && fabsf(kxf) < kcut && fabsf(kyf) < kcut) {
        // both squares rounded before the sum (no multiply-add contraction), as the
        // reference's f32 expression is written; the scalings are exact
        const float ensf = 0.5f * __fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)) * inv_n4f;
        const float enef = ensf / k2f;
        const int fb = (int)min((uint32_t)fb_raw, (uint32_t)(nb - 1));
        if (fb != cur_fb) {
          if (cur_fb >= 0) atomicAdd(&fhist[cur_fb], cur_f);
          cur_fb = fb;
          cur_f = 0u;
        }
        cur_f += (uint32_t)(enef * 1e8f);
        fe += (uint32_t)(enef * 1e6f);
        fz += (uint32_t)(ensf * 1e6f);
      }
    }
    if (cur_b >= 0) {
      const unsigned r = (unsigned)(cur_b - lo);
      if (r < (unsigned)kDiagSpan) atomicAdd(my + r, cur_e);
      else atomicAdd(out + cur_b, cur_e);
    }
    if (cur_fb >= 0) atomicAdd(&fhist[cur_fb], cur_f);
  }
  ene = warp_sum(ene);
  ens = warp_sum(ens);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    fe += __shfl_xor_sync(0xffffffffu, fe, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (lane == 0) {
    atomicAdd(&tot[0], ene);
    atomicAdd(&tot[1], ens);
    atomicAdd(&fhist[nb], fe);
    atomicAdd(&fhist[nb + 1], fz);
  }
  __syncthreads();
  // window bin r summed over the 32 lanes' windows in a fixed order: thread (g, r) adds
  // lanes [11 g, 11 g + 11) of bin r and leaves the sum in the slot of lane 11 g (no other
  // thread reads or writes bin r of those lanes), then thread r adds the three partials
  static_assert(3 * kDiagSpan <= 256, "three partial sums per window bin");
  if ((int)threadIdx.x < 3 * kDiagSpan) {
    const int g = (int)threadIdx.x / kDiagSpan, r = (int)threadIdx.x - g * kDiagSpan;
    const int l0 = 11 * g, l1 = min(l0 + 11, 32);
    double v = win[l0 * kDiagStride + r];
    for (int l = l0 + 1; l < l1; ++l) v += win[l * kDiagStride + r];
    win[l0 * kDiagStride + r] = v;
  }
  __syncthreads();
  if ((int)threadIdx.x < kDiagSpan) {
    const int r = (int)threadIdx.x;
    const double v = (win[r] + win[11 * kDiagStride + r]) + win[22 * kDiagStride + r];
    if (v != 0.0 && lo + r < nb) atomicAdd(&out[lo + r], v);
  }
  if (threadIdx.x == 0) {
    atomicAdd(&out[nb], tot[0]);
    atomicAdd(&out[nb + 1], tot[1]);
  }
  for (int i = threadIdx.x; i < nb + 2; i += blockDim.x)
    if (fhist[i] != 0u) atomicAdd(&bins[i], fhist[i]);
}

// ------------------------------------------------------------------ scenarios
// SCENARIOS[kind].build(n, cfg) of scenarios.js, evaluated per cell in FP64 and
// rounded to FP32 (the reference's Float32Array).  Grid: x = col h, y = row h,
// h = 2 pi / n (scenarios.js:3-13).
__device__ __forceinline__ double scen_wrap_delta(double a, double b) {   // scenarios.js:20-28
  constexpr double kPi = 3.14159265358979323846, k2Pi = 2.0 * kPi;
  double d = a - b;
  if (d > kPi) d -= k2Pi;
  else if (d < -kPi) d += k2Pi;
  return d;
}
// one Gaussian blob of blobs() (scenarios.js:30-44)
__device__ __forceinline__ double scen_blob(double x, double y, double bx, double by, double a, double amp) {
  const double dx = scen_wrap_delta(x, bx), dy = scen_wrap_delta(y, by);
  const double r2 = dx * dx + dy * dy, s2 = a * a;
  return r2 < 25.0 * s2 ? amp * exp(-r2 / s2) : 0.0;
}
__global__ void k_scenario(float* out, int n, int kind, double param) {
  constexpr double kPi = 3.14159265358979323846, k2Pi = 2.0 * kPi;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  const int row = idx / n, col = idx - row * n;
  const double h = k2Pi / n;
  const double x = col * h, y = row * h;
  double v = 0.0;
  switch (kind) {
    case 0: {   // 'shear layer' (scenarios.js:70-79)
      const double delta = fmax(k2Pi / 30.0, (6.0 * k2Pi) / n);
      const double eps = 0.05;
      const bool lower = y <= kPi;
      const double z = lower ? (y - kPi / 2.0) / delta : (1.5 * kPi - y) / delta;
      const double c = cosh(z);
      const double dudy = ((lower ? 1.0 : -1.0) * (1.0 / (c * c))) / delta;
      v = eps * cos(x) - dudy;
      break;
    }
    case 1:     // 'taylor-green' (scenarios.js:94-97)
      v = 6.0 * cos(2.0 * x) * cos(2.0 * y);
      break;
    case 2: {   // dipole (scenarios.js:112-122)
      const double gamma = 12.0, a = 0.3, d = 0.9;
      const double amp = gamma / (kPi * a * a), cx = kPi * 0.6;
      v = scen_blob(x, y, cx, kPi - d / 2.0, a, amp);
      v += scen_blob(x, y, cx, kPi + d / 2.0, a, -amp);
      break;
    }
    case 3: {   // merger (scenarios.js:136-143), d = cfg.mergerSep
      const double a = 0.22, d = param;
      v = scen_blob(x, y, kPi - d / 2.0, kPi, a, 30.0);
      v += scen_blob(x, y, kPi + d / 2.0, kPi, a, 30.0);
      break;
    }
    default: {  // polygon: ring(n, round(cfg.polygonN), 1.25, 0.19, 34, 0.02) (scenarios.js:46-56,157-159)
      const int count = (int)floor(param + 0.5);
      const double radius = 1.25, a = 0.19, amp = 34.0, jitter = 0.02;
      const int mode = max(2, count / 2);
      for (int j = 0; j < count; ++j) {
        const double th = (k2Pi * j) / count;
        const double r = radius * (1.0 + jitter * cos((k2Pi * mode * j) / count));
        v += scen_blob(x, y, kPi + r * cos(th), kPi + r * sin(th), a, amp);
      }
      break;
    }
  }
  out[idx] = (float)v;
}

// ------------------------------------------------------------------ dye
// JS toHalf (solver.js:20-41): f32 -> binary16 by mantissa truncation
__device__ __forceinline__ uint16_t to_half_trunc(float value) {
  const uint32_t x = __float_as_uint(value);
  const uint32_t sign = (x >> 16) & 0x8000u;
  int exp = (int)((x >> 23) & 0xffu);
  uint32_t mant = x & 0x7fffffu;
  if (exp == 255) return (uint16_t)(sign | 0x7c00u | (mant ? 0x200u : 0u));
  exp = exp - 127 + 15;
  if (exp >= 31) return (uint16_t)(sign | 0x7c00u);
  if (exp <= 0) {
    if (exp < -10) return (uint16_t)sign;
    mant = (mant | 0x800000u) >> (1 - exp);
    return (uint16_t)(sign | (mant >> 13));
  }
  return (uint16_t)(sign | ((uint32_t)exp << 10) | (mant >> 13));
}

// 'bands' pattern (solver.js:450-466), computed in double like the JS
__global__ void k_paint_bands(ushort4* dye, int m) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= m * m) return;
  const int row = idx / m, col = idx % m;
  const double fy = (double)row / m, fx = (double)col / m;
  const double band = 0.5 + 0.5 * tanh(6.0 * sin(fy * 3.14159265358979323846 * 12.0));
  const double mix = 0.5 + 0.5 * sin(fx * 3.14159265358979323846 * 2.0);
  const double warm[3] = {1.0, 0.45, 0.22}, cool[3] = {0.28, 0.62, 1.0};
  uint16_t c[3];
  for (int k = 0; k < 3; ++k) c[k] = to_half_trunc((float)(band * (warm[k] * mix + cool[k] * (1.0 - mix)) * 0.9));
  dye[idx] = make_ushort4(c[0], c[1], c[2], to_half_trunc(1.0f));
}

}  // namespace s2d
