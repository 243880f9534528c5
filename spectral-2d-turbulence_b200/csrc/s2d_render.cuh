// s2d_render.cuh -- headless image of the solver state: the arithmetic of the
// reference's fragment shader (render.wgsl:81-103, modes of render.js:4) as a CUDA
// kernel writing an RGBA8 buffer instead of a swapchain image.
#pragma once
#include "s2d_dye.cuh"

namespace s2d {

__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.f - t) + b * t; }
__device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {   // WGSL smoothstep
  const float t = fminf(fmaxf((x - e0) / (e1 - e0), 0.f), 1.f);
  return t * t * (3.f - 2.f * t);
}
__device__ __forceinline__ float3 vort_color(float t) {                       // render.wgsl:61-72
  const float a = fminf(fmaxf(t, -1.f), 1.f), m = fabsf(a);
  const float3 hue = a > 0.f ? make_float3(1.00f, 0.40f, 0.12f) : make_float3(0.16f, 0.52f, 1.00f);
  const float s = smoothstepf(0.f, 0.60f, m);
  const float3 base = make_float3(mixf(0.035f, hue.x, s), mixf(0.042f, hue.y, s), mixf(0.062f, hue.z, s));
  const float w = smoothstepf(0.70f, 1.f, m) * 0.7f;
  return make_float3(mixf(base.x, 1.0f, w), mixf(base.y, 0.95f, w), mixf(base.z, 0.88f, w));
}
__device__ __forceinline__ float3 heat(float t) {                              // render.wgsl:74-80
  const float x = fminf(fmaxf(t, 0.f), 1.f);
  const float r = fminf(fmaxf(1.55f * x - 0.18f, 0.f), 1.f);
  const float g = fminf(fmaxf(1.32f * x * x - 0.06f, 0.f), 1.f);
  const float b = fminf(fmaxf(2.20f * x * x * x * (1.f - 0.55f * x) + 0.14f * x, 0.f), 1.f);
  return make_float3(r * 0.94f + 0.03f, g * 0.94f + 0.035f, b * 0.94f + 0.055f);
}
__device__ __forceinline__ unsigned char to_unorm8(float c) {
  return (unsigned char)__float2int_rn(fminf(fmaxf(c, 0.f), 1.f) * 255.f);
}

// out: height x width RGBA8, row 0 = top of the image (uv.y = 1 - (row + 0.5)/height,
// the fragment's uv for a full-screen triangle, render.wgsl:27-34); omega: physical
// vorticity (float2, .x) on the n x n grid; vel: (u, v); dye: m x m binary16 texels
__global__ void k_render(uchar4* out, int width, int height, const float2* __restrict__ omega,
                         const float2* __restrict__ vel, const uint2* __restrict__ dye, int n, int m, int mode,
                         float exposure, float vort_scale, float dye_gain) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= width || py >= height) return;
  const float u = (px + 0.5f) / width, v = 1.f - (py + 0.5f) / height;
  const Rgba d = bilerp(GlobalTex{dye, m}, footprint(u, v, m));
  const float3 dy = make_float3(d.r * dye_gain, d.g * dye_gain, d.b * dye_gain);
  const float om = sample_vel(GlobalVel{omega, n}, u, v, n).x;
  const float t = fminf(fmaxf(om * vort_scale, -1.f), 1.f);
  float3 col;
  if (mode == 0) {
    col = dy;
  } else if (mode == 1) {
    col = vort_color(t);
  } else if (mode == 2) {
    const float3 sh = vort_color(t);
    const float a = 0.30f + 0.70f * exposure, b = 0.55f + 0.45f * fabsf(t);
    col = make_float3(sh.x * a + dy.x * b, sh.y * a + dy.y * b, sh.z * a + dy.z * b);
  } else {
    const float2 w = sample_vel(GlobalVel{vel, n}, u, v, n);
    col = heat(sqrtf(w.x * w.x + w.y * w.y) * vort_scale * 0.75f);
  }
  col = make_float3(1.f - expf(-col.x * exposure), 1.f - expf(-col.y * exposure), 1.f - expf(-col.z * exposure));
  auto g = [](float c) { return powf(fminf(fmaxf(c, 0.f), 1.f), 0.4545f); };
  out[(size_t)py * width + px] = make_uchar4(to_unorm8(g(col.x)), to_unorm8(g(col.y)), to_unorm8(g(col.z)), 255);
}

}  // namespace s2d
