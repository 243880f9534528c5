// s2d_band.cuh -- band-limited Gaussian initial spectra (benchmark initial condition).
#pragma once
#include "s2d_device.cuh"

namespace s2d {

// Complex standard Gaussian for spectral cell `idx` of a stream `seed`:
// Box-Muller over two hash1 draws (counter-based, order independent).
__device__ __forceinline__ float2 gauss_cell(uint32_t seed, uint32_t idx) {
  const uint32_t h1 = hash1(idx ^ hash1(seed ^ 0x68bc21ebu));
  const uint32_t h2 = hash1(h1 ^ 0x02e5be93u);
  const double u1 = ((double)h1 + 0.5) * (1.0 / 4294967296.0);
  const double u2 = (double)h2 * (1.0 / 4294967296.0);
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  return make_float2((float)(r * c), (float)(r * s));
}

// Band value at (row, col) of an n x n grid: w(k) = (g(k) + conj g(-k)) / 2 inside
// kmin <= |k| <= kmax and the 2/3 band, zero elsewhere and at k = 0.
__device__ __forceinline__ float2 band_cell(uint32_t seed, int n, int row, int col, float kmin, float kmax) {
  const float kx = wn_rt(col, n), ky = wn_rt(row, n);
  const float kr = sqrtf(kx * kx + ky * ky);
  const float kcut = (float)(n / 3.0);
  if (kr == 0.f || kr < kmin || kr > kmax || !(fabsf(kx) < kcut && fabsf(ky) < kcut)) return make_float2(0.f, 0.f);
  const int prow = (n - row) & (n - 1), pcol = (n - col) & (n - 1);
  const float2 a = gauss_cell(seed, (uint32_t)(row * n + col));
  const float2 b = gauss_cell(seed, (uint32_t)(prow * n + pcol));
  return make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
}

}  // namespace s2d
