// s2d_device.cuh -- device-side parameter blocks and per-cell helpers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "fft_core.cuh"

namespace s2d {

constexpr float kTwoPiF = 6.28318530717958647f;  // TWO_PI, common.wgsl:5

// Params uniform of the reference (common.wgsl:8-21), plus the grid constants
// the reference templates into each shader (shaders.js:20-28).  Lives in
// device memory; written by configure(), read by every stage kernel.
struct DevParams {
  float beta, mu, nu_h;
  int32_t hyper_p;
  float force_amp, force_k, force_width;
  uint32_t step_index;
  float dx, cfl, dt_min, dt_max;
  float dye_fade, kcut, force_norm;
  int32_t n;
};

// Splat / Splats uniform (common.wgsl:23-40)
struct DevSplat {
  float x, y, vx, vy;
  float r, g, b, radius;
  float amp, dye_amp, pad0, pad1;
};
struct DevSplats {
  int32_t count, pad0, pad1, pad2;
  DevSplat items[8];
};

// RK3 coefficient rows [cA, a, cB, b] (solver.js:11-15)
__host__ __device__ constexpr float rk_cA(int s) { return s == 0 ? 0.f : s == 1 ? 0.75f : 1.f / 3.f; }
__host__ __device__ constexpr float rk_cB(int s) { return s == 0 ? 1.f : s == 1 ? 0.25f : 2.f / 3.f; }
__host__ __device__ constexpr float rk_a(int s) { return s == 0 ? 0.f : s == 1 ? 0.5f : 1.f; }
__host__ __device__ constexpr float rk_b(int s) { return s == 0 ? 1.f : s == 1 ? -0.5f : 0.5f; }

// signed wavenumber of FFT index i (common.wgsl:50-55)
template <int N> __device__ __forceinline__ float wn(int i) { return (float)(i < N / 2 ? i : i - N); }
__device__ __forceinline__ float wn_rt(int i, int n) { return (float)(i < n / 2 ? i : i - n); }

// PCG-style hash (common.wgsl:76-80) and its unit float (common.wgsl:82-84)
__host__ __device__ __forceinline__ uint32_t hash1(uint32_t x) {
  uint32_t v = x * 747796405u + 2891336453u;
  v = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
  return (v >> 22u) ^ v;
}
__device__ __forceinline__ float hashf(uint32_t a, uint32_t b) {
  return __uint2float_rn(hash1(a ^ hash1(b))) * 2.3283064365386963e-10f;
}

// k^(2p) as (k2)^p for integer p >= 0: ((k2 k2) k2) ... left to right, unrolled up
// to p = 8 (the viscosity orders used) with a loop beyond
__device__ __forceinline__ float powi(float k2, int p) {
  float r = 1.f;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if (i < p) r *= k2;
  for (int i = 8; i < p; ++i) r *= k2;
  return r;
}

// k2 outside [lo2, hi2] has forcing envelope exp(-((|k| - K)/W)^2) below 1e-4, the
// reference's cut: |(|k| - K)/W| > 3.05 > sqrt(ln 1e4) = 3.035 (a conservative
// pre-test; cells inside run the exact test)
__device__ __forceinline__ float2 forcing_k2_bounds(const DevParams& P) {
  const float lo = fmaxf(P.force_k - 3.05f * fabsf(P.force_width), 0.f);
  const float hi = P.force_k + 3.05f * fabsf(P.force_width);
  return make_float2(lo * lo, hi * hi);
}

// White-in-time stochastic forcing of one spectral cell (solver.wgsl:77-92).
// Caller guarantees the cell is in the dealias band with k2 > 0.
__device__ __forceinline__ float2 stochastic_term(const DevParams& P, int n, int row, int col, float kx,
                                                  float ky, float k2, float dt) {
  const float d = (sqrtf(k2) - P.force_k) / P.force_width;
  const float env = expf(-(d * d));
  if (!(env > 1e-4f)) return make_float2(0.f, 0.f);
  const bool canon = ky > 0.f || (ky == 0.f && kx > 0.f);
  const uint32_t hr = canon ? (uint32_t)row : (uint32_t)((n - row) & (n - 1));
  const uint32_t hc = canon ? (uint32_t)col : (uint32_t)((n - col) & (n - 1));
  const float sgn = canon ? 1.f : -1.f;
  const float ph = kTwoPiF * hashf(hr * (uint32_t)n + hc, P.step_index);
  const float amp = P.force_amp * env * P.force_norm / sqrtf(fmaxf(dt, 1e-6f));
  float s, c;
  sincosf(ph, &s, &c);
  return make_float2(amp * c, sgn * amp * s);
}

// Integrating factor over half a step, carried as E(dt/2) - 1 so that factors
// close to one keep their full relative precision: E = exp(L dt/2) with
// L = -mu - nu_h k2^p + i beta kx/k2 (solver.wgsl:97-101, spectral2d.py:26).
// exp(x) for |x| ~ 1e-5 rounded to FP32 keeps only ~3 digits of 1 - E, which
// biases the damping by ~1e-5 per hundred steps; expm1 and the half-angle form
// cos(t) - 1 = -2 sin^2(t/2) avoid the cancellation.
//
// e^x - 1: for |x| < 1/4 the Taylor series to x^7/7! (truncation below
// |x|^7/8! < 1.5e-9 relative), else expf(x) - 1, which has no cancellation there
// (|e^x - 1| >= 0.22) and saturates to -1 / overflows to inf like expm1.
__device__ __forceinline__ float expm1_series(float x) {
  if (fabsf(x) < 0.25f) {
    float p = 1.f / 5040.f;
    p = fmaf(p, x, 1.f / 720.f);
    p = fmaf(p, x, 1.f / 120.f);
    p = fmaf(p, x, 1.f / 24.f);
    p = fmaf(p, x, 1.f / 6.f);
    p = fmaf(p, x, 0.5f);
    p = fmaf(p, x, 1.f);
    return p * x;
  }
  return expf(x) - 1.f;
}
// sin and cos of a: Taylor series for |a| <= pi/4 (sin to a^9/9!, cos to a^10/10!;
// truncation below 3e-9 relative), sincosf beyond.
__device__ __forceinline__ void sincos_series(float a, float* s, float* c) {
  if (fabsf(a) <= 0.78539816f) {
    const float a2 = a * a;
    float ps = 1.f / 362880.f;
    ps = fmaf(ps, a2, -1.f / 5040.f);
    ps = fmaf(ps, a2, 1.f / 120.f);
    ps = fmaf(ps, a2, -1.f / 6.f);
    ps = fmaf(ps, a2, 1.f);
    float pc = -1.f / 3628800.f;
    pc = fmaf(pc, a2, 1.f / 40320.f);
    pc = fmaf(pc, a2, -1.f / 720.f);
    pc = fmaf(pc, a2, 1.f / 24.f);
    pc = fmaf(pc, a2, -0.5f);
    *s = ps * a;
    *c = fmaf(pc, a2, 1.f);
    return;
  }
  sincosf(a, s, c);
}
__device__ __forceinline__ float2 half_factor_m1(const DevParams& P, float kx, float k2, float dt) {
  const float re = -P.mu - P.nu_h * powi(k2, P.hyper_p);
  const float d = expm1_series(re * (0.5f * dt));
  if (P.beta == 0.f) return make_float2(d, 0.f);
  const float th = P.beta * __fdividef(kx, k2) * (0.5f * dt);
  float sh, ch;
  sincos_series(0.5f * th, &sh, &ch);
  const float g = -2.f * sh * sh;         // cos(th) - 1
  const float sn = 2.f * sh * ch;         // sin(th)
  return make_float2(d + g + d * g, (1.f + d) * sn);
}

// (1 + e) * w without forming 1 + e; a zero w stays zero even when e overflows
// (the reference's E * 0 with E = inf gives NaN at modes outside the band).
__device__ __forceinline__ float2 apply_m1(float2 e, float2 w) {
  if (w.x == 0.f && w.y == 0.f) return w;
  const float2 ew = cmul(e, w);
  return make_float2(w.x + ew.x, w.y + ew.y);
}

// wout = cA E(a dt) w0 + cB E(b dt) (wcur + dt rhs) for stage s, from e = E(dt/2) - 1:
// E(dt) - 1 = e (2 + e), E(-dt/2) - 1 = -e / (1 + e)  (one expm1 and one sincos per cell).
template <int S>
__device__ __forceinline__ float2 rk_update(float2 e, float2 w0, float2 wcur, float2 rhs, float dt) {
  const float2 adv = make_float2(wcur.x + dt * rhs.x, wcur.y + dt * rhs.y);
  if constexpr (S == 0) {
    const float2 full = cmul(e, make_float2(2.f + e.x, e.y));
    return apply_m1(full, adv);
  } else if constexpr (S == 1) {
    const float2 one_e = make_float2(1.f + e.x, e.y);
    const float rden = __frcp_rn(one_e.x * one_e.x + one_e.y * one_e.y);
    const float2 q = cmul(e, cconj(one_e));
    const float2 mhalf = make_float2(-q.x * rden, -q.y * rden);
    const float2 a = apply_m1(e, w0), b = apply_m1(mhalf, adv);
    return make_float2(0.75f * a.x + 0.25f * b.x, 0.75f * a.y + 0.25f * b.y);
  } else {
    // 1/3 a + 2/3 b as b + (a - b)/3: the FP32 constants 1/3 and 2/3 both round up
    // (their sum is 1 + 3e-8), which would bias every step; on (a - b) the bias vanishes
    const float2 full = cmul(e, make_float2(2.f + e.x, e.y));
    const float2 a = apply_m1(full, w0), b = apply_m1(e, adv);
    return make_float2(b.x + (a.x - b.x) * (1.f / 3.f), b.y + (a.y - b.y) * (1.f / 3.f));
  }
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// periodic helpers of common.wgsl:42-48
__device__ __forceinline__ float wrap01(float x) { return x - floorf(x); }
__device__ __forceinline__ float sepf(float a, float b) { return wrap01(a - b + 0.5f) - 0.5f; }

// CFL dt from the maximum of |u|+|v| (reduce.wgsl:54-62)
__device__ __forceinline__ float cfl_dt(const DevParams& P, float speed) {
  float dt = P.dt_max;
  if (speed > 1e-8f) dt = fminf(P.dt_max, P.cfl * P.dx / speed);
  return fmaxf(dt, P.dt_min);
}

}  // namespace s2d
