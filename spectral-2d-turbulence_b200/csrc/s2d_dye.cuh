// s2d_dye.cuh -- BFECC + MacCormack-limited semi-Lagrangian dye advection (dye.wgsl).
//
// The dye is M x M rgba16float texels (ushort4 of binary16 bits) on a grid
// refined dyeScale times over the N x N velocity grid.  Texture filtering is
// restated in software: repeat-wrapped bilinear in FP32 (the reference samples
// with a linear-filtered, repeat-addressed sampler).
//
// Two implementations share every sampling function, so they agree bit for bit:
//   * three passes (advect_fwd, advect_back, advect_corr) exactly as the
//     reference dispatches them, each reading and writing whole textures;
//   * k_dye_fused: one launch per step.  A CTA owns a TX x 32 output tile (TX = 64,
//     or 32 when the dye is not refined over the flow) and keeps, in shared memory,
//     the source texels of the tile plus a 3-level halo, the forward-pass texels of
//     the tile plus 2 levels and the backward-pass texels plus 1 level; each level's
//     halo (1 texel on each side) covers the bilinear footprint of a trace shorter than
//     one texel, which the CFL limit gives at dyeScale 2 away from the fastest flow.  A
//     sample outside the on-chip region is recomputed from global memory (the
//     forward/backward values at that texel are re-derived), so the result does not
//     depend on the halo being large enough.  Texture traffic drops from 7 texture
//     passes to one read and one write.  The source, forward and backward windows hold
//     binary16 texels, as those textures would (exact), and only r, g, b are carried:
//     the corrected texel's alpha is 1 whatever the inputs.
#pragma once
#include <cuda_fp16.h>
#include "s2d_device.cuh"

namespace s2d {

struct Rgba {
  float r, g, b, a;
};

__device__ __forceinline__ Rgba unpack_texel(uint2 u) {
  const float2 rg = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
  const float2 ba = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
  return {rg.x, rg.y, ba.x, ba.y};
}
__device__ __forceinline__ uint2 pack_texel(float r, float g, float b, float a) {
  const __half2 rg = __floats2half2_rn(r, g), ba = __floats2half2_rn(b, a);
  return make_uint2(*reinterpret_cast<const unsigned*>(&rg), *reinterpret_cast<const unsigned*>(&ba));
}
__device__ __forceinline__ Rgba round_texel(const Rgba& c) { return unpack_texel(pack_texel(c.r, c.g, c.b, c.a)); }

// ---------------------------------------------------------------- fetchers
struct GlobalTex {
  const uint2* t;
  int m;
  __device__ __forceinline__ Rgba operator()(int x, int y) const { return unpack_texel(__ldg(t + (size_t)y * m + x)); }
};
struct GlobalVel {
  const float2* v;
  int n;
  __device__ __forceinline__ float2 operator()(int x, int y) const { return __ldg(v + (size_t)y * n + x); }
};

// Every operation below is an explicitly rounded intrinsic (no multiply-add
// contraction), so the fused and the three-pass kernels produce the same bits.  Where a
// product is exact -- a coordinate in [0, 1] times the power-of-two grid size -- the
// multiply and the following add are one fused multiply-add with the same result.
__device__ __forceinline__ float lerp1(float a, float b, float t) {
  return __fmaf_rn(b, t, __fmul_rn(a, __fsub_rn(1.f, t)));   // WGSL mix(a, b, t)
}
// lerp1 on two channels at once with the packed FP32x2 pipe (sm_100): each lane is the
// same correctly rounded multiply and fused multiply-add, so the bits equal lerp1's
__device__ __forceinline__ float2 lerp2v(float2 a, float2 b, float t) {
  const float omt = __fsub_rn(1.f, t);
  return __ffma2_rn(b, make_float2(t, t), __fmul2_rn(a, make_float2(omt, omt)));
}

// bilinear velocity at normalised p (dye.wgsl:27-38); cell indices wrapped
template <class VF>
__device__ __forceinline__ float2 sample_vel(const VF& vf, float px, float py, int n) {
  const float nf = (float)n;
  const float gx = __fmaf_rn(px, nf, -0.5f), gy = __fmaf_rn(py, nf, -0.5f);   // px * nf exact
  const float bx = floorf(gx), by = floorf(gy);
  const float fx = __fsub_rn(gx, bx), fy = __fsub_rn(gy, by);
  const int ix = (int)bx, iy = (int)by;
  const int x0 = ix & (n - 1), x1 = (ix + 1) & (n - 1), y0 = iy & (n - 1), y1 = (iy + 1) & (n - 1);
  const float2 v00 = vf(x0, y0), v10 = vf(x1, y0), v01 = vf(x0, y1), v11 = vf(x1, y1);
  return lerp2v(lerp2v(v00, v10, fx), lerp2v(v01, v11, fx), fy);
}

// midpoint back-trace (dye.wgsl:40-45), from the velocity v1 already sampled at p
// (0.5 (v h) is v (h/2): halving commutes with the rounding of the product)
// fract(p - v s + 1) on both coordinates with the packed pipe, as fract(p - d + 1) with
// d = v s rounded: p - d is p + (-d), and the negation is exact.  The product is rounded
// before the sum: it is formed as a fused multiply-add with a +0 addend, which no compiler
// may turn back into a multiply (it differs from one in the sign of a zero product) and so
// into a multiply-add with p.  A packed multiply followed by a packed add -- __fmul2_rn /
// __fadd2_rn, and PTX mul.rn / add.rn on f32x2 alike -- was measured contracted into one
// FFMA2 (one FP32 unit apart in ~1e-4 of the trace positions).  p is a texel centre, never
// zero, so p + (+0) is p.
__device__ __forceinline__ float2 fract_shift2(float2 p, float2 v, float s) {
  const float2 d = __ffma2_rn(v, make_float2(-s, -s), make_float2(0.f, 0.f));
  const float2 x = __fadd2_rn(__fadd2_rn(p, d), make_float2(1.f, 1.f));
  return make_float2(__fsub_rn(x.x, floorf(x.x)), __fsub_rn(x.y, floorf(x.y)));
}
template <class VF>
__device__ __forceinline__ float2 trace_from(const VF& vf, float px, float py, float2 v1, float h, int n) {
  const float hh = 0.5f * h;
  const float2 p = make_float2(px, py);
  const float2 mid = fract_shift2(p, v1, hh);
  const float2 v2 = sample_vel(vf, mid.x, mid.y, n);
  return fract_shift2(p, v2, h);
}
template <class VF>
__device__ __forceinline__ float2 trace_pos(const VF& vf, float px, float py, float h, int n) {
  return trace_from(vf, px, py, sample_vel(vf, px, py, n), h, n);
}

// texel footprint of a repeat-addressed linear sample at normalised s
struct Footprint {
  int x0, x1, y0, y1;
  float fx, fy;
};
__device__ __forceinline__ Footprint footprint(float sx, float sy, int m) {
  const float mf = (float)m;
  const float gx = __fmaf_rn(sx, mf, -0.5f), gy = __fmaf_rn(sy, mf, -0.5f);   // sx * mf exact
  const float bx = floorf(gx), by = floorf(gy);
  Footprint f;
  f.fx = __fsub_rn(gx, bx);
  f.fy = __fsub_rn(gy, by);
  f.x0 = (int)bx & (m - 1);
  f.x1 = ((int)bx + 1) & (m - 1);
  f.y0 = (int)by & (m - 1);
  f.y1 = ((int)by + 1) & (m - 1);
  return f;
}

__device__ __forceinline__ float lerp2(float a00, float a10, float a01, float a11, float fx, float fy) {
  return lerp1(lerp1(a00, a10, fx), lerp1(a01, a11, fx), fy);
}

template <class TF>
__device__ __forceinline__ Rgba bilerp(const TF& tf, const Footprint& f, Rgba* lo = nullptr, Rgba* hi = nullptr) {
  const Rgba c00 = tf(f.x0, f.y0), c10 = tf(f.x1, f.y0), c01 = tf(f.x0, f.y1), c11 = tf(f.x1, f.y1);
  if (lo) {
    lo->r = fminf(fminf(c00.r, c10.r), fminf(c01.r, c11.r));
    lo->g = fminf(fminf(c00.g, c10.g), fminf(c01.g, c11.g));
    lo->b = fminf(fminf(c00.b, c10.b), fminf(c01.b, c11.b));
    hi->r = fmaxf(fmaxf(c00.r, c10.r), fmaxf(c01.r, c11.r));
    hi->g = fmaxf(fmaxf(c00.g, c10.g), fmaxf(c01.g, c11.g));
    hi->b = fmaxf(fmaxf(c00.b, c10.b), fmaxf(c01.b, c11.b));
  }
  const float2 rg = lerp2v(lerp2v(make_float2(c00.r, c00.g), make_float2(c10.r, c10.g), f.fx),
                           lerp2v(make_float2(c01.r, c01.g), make_float2(c11.r, c11.g), f.fx), f.fy);
  const float2 ba = lerp2v(lerp2v(make_float2(c00.b, c00.a), make_float2(c10.b, c10.a), f.fx),
                           lerp2v(make_float2(c01.b, c01.a), make_float2(c11.b, c11.a), f.fx), f.fy);
  return {rg.x, rg.y, ba.x, ba.y};
}

// texel centre (x + 0.5)/m; m is a power of two, so x/m, 0.5/m and their sum (2x+1)/(2m)
// are all exact and one fused multiply-add gives the quotient
__device__ __forceinline__ float2 texel_pos(int x, int y, float inv_m) {
  const float half_inv = 0.5f * inv_m;
  return make_float2(__fmaf_rn((float)x, inv_m, half_inv), __fmaf_rn((float)y, inv_m, half_inv));
}
__device__ __forceinline__ float2 texel_pos(int x, int y, int m) { return texel_pos(x, y, __frcp_rn((float)m)); }

// BFECC correction of one texel from its source (a, with the 4-texel min/max) and
// back-advected (b) samples, fade and splat dye (dye.wgsl:81-112); pos() gives the texel
// centre, formed only when there are splats to place
template <class POS>
__device__ __forceinline__ uint2 correct_from(const Rgba& a, const Rgba& b, const Rgba& lo, const Rgba& hi,
                                              const POS& pos, float fade, const DevSplats* __restrict__ S) {
  auto corr = [&](float x, float y, float l, float u) {
    return __fmul_rn(fminf(fmaxf(__fsub_rn(__fmul_rn(1.5f, x), __fmul_rn(0.5f, y)), l), u), fade);
  };
  float r = corr(a.r, b.r, lo.r, hi.r);
  float g = corr(a.g, b.g, lo.g, hi.g);
  float bb = corr(a.b, b.b, lo.b, hi.b);
  const int cnt = S->count;
  if (cnt == 0) return pack_texel(r, g, bb, 1.f);
  const float2 p = pos();
  const float px = p.x, py = p.y;
  for (int i = 0; i < cnt; ++i) {
    const DevSplat sp = S->items[i];
    const float rx = sepf(px, sp.x), ry = sepf(py, sp.y);
    const float sig2 = fmaxf(__fmul_rn(sp.radius, sp.radius), 1e-8f);
    const float r2 = __fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry));
    if (r2 < __fmul_rn(9.f, sig2)) {
      const float wgt = __fmul_rn(sp.dye_amp, expf(-__fdiv_rn(r2, sig2)));
      r = __fadd_rn(r, __fmul_rn(sp.r, wgt));
      g = __fadd_rn(g, __fmul_rn(sp.g, wgt));
      bb = __fadd_rn(bb, __fmul_rn(sp.b, wgt));
    }
  }
  return pack_texel(r, g, bb, 1.f);
}

template <class SF, class BF>
__device__ __forceinline__ uint2 correct_texel(const SF& src, const BF& back, const Footprint& f, float px, float py,
                                               float fade, const DevSplats* __restrict__ S) {
  Rgba lo, hi;
  const Rgba a = bilerp(src, f, &lo, &hi);
  const Rgba b = bilerp(back, f);
  return correct_from(a, b, lo, hi, [&] { return make_float2(px, py); }, fade, S);
}

// ---------------------------------------------------------------- three passes (reference order)
// advect_fwd / advect_back (dye.wgsl:58-74): dst = src sampled at trace(p, sign*dt/2pi)
__global__ void k_dye_advect(const float2* __restrict__ vel, const uint2* __restrict__ src, uint2* dst,
                             const float* __restrict__ dtbuf, float sign, int n, int m) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
  if (gx >= m || gy >= m) return;
  const float2 p = texel_pos(gx, gy, m);
  const float h = __fdiv_rn(__fmul_rn(sign, dtbuf[0]), kTwoPiF);
  const float2 s = trace_pos(GlobalVel{vel, n}, p.x, p.y, h, n);
  const Rgba c = bilerp(GlobalTex{src, m}, footprint(s.x, s.y, m));
  dst[(size_t)gy * m + gx] = pack_texel(c.r, c.g, c.b, c.a);
}

// advect_corr (dye.wgsl:76-113)
__global__ void k_dye_correct(const float2* __restrict__ vel, const uint2* __restrict__ src,
                              const uint2* __restrict__ aux, uint2* dst, const float* __restrict__ dtbuf,
                              const DevParams* __restrict__ params, const DevSplats* __restrict__ S, int n, int m) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
  if (gx >= m || gy >= m) return;
  const float2 p = texel_pos(gx, gy, m);
  const float h = __fdiv_rn(dtbuf[0], kTwoPiF);
  const float2 s = trace_pos(GlobalVel{vel, n}, p.x, p.y, h, n);
  dst[(size_t)gy * m + gx] =
      correct_texel(GlobalTex{src, m}, GlobalTex{aux, m}, footprint(s.x, s.y, m), p.x, p.y, params->dye_fade, S);
}

// ---------------------------------------------------------------- fused single pass
// Halo per level: a sample displaced by less than one texel from the centre of texel x
// (floor(x + d) is x - 1 or x for |d| < 1) has the bilinear footprint [x - 1, x + 1], so
// each level extends the region by one texel on each side.
constexpr int kDyeLo = 1, kDyeHi = 1;
constexpr int kDyeTileY = 32;
// Output tile TX x 32 (TX = 64 when the dye is refined over the flow: 103 KB of windows,
// 2 CTAs of 512 threads per SM, and 20 % / 10 % of recomputed forward / backward halo
// texels instead of 28 % / 14 % at TX = 32; TX = 32 otherwise, where the velocity window
// is as large as the dye windows)
template <int TX> struct DyeGeom {
  static constexpr int TY = kDyeTileY;
  static constexpr int THREADS = TX * 8;
  static constexpr int MINB = TX >= 64 ? 2 : 3;   // resident CTAs per SM (shared memory bound)
  static constexpr int H = kDyeLo + kDyeHi;
  static constexpr int W1X = TX + H, W1Y = TY + H;           // backward-pass region
  static constexpr int W2X = TX + 2 * H, W2Y = TY + 2 * H;   // forward-pass region
  // source region, widened by one texel below (and one above, for an even width) so that
  // its rows start on an even texel and arrive in 16-byte copies
  static constexpr int W3X = (TX + 3 * H + 2) & ~1, W3Y = TY + 3 * H;
  static_assert(W3X % 2 == 0 && TX % 2 == 0, "16-byte source rows");
  // velocity cells needed by traces from the forward-pass region, for an n x n velocity
  // grid under an m x m dye grid: (W2 + 2 displacement texels) * n/m + 2 interpolation /
  // rounding cells on each side
  __host__ __device__ static constexpr int vel_x(int n, int m) { return (W2X + 2) * n / m + 4; }
  __host__ __device__ static constexpr int vel_y(int n, int m) { return (W2Y + 2) * n / m + 4; }
  // binary16 source / backward / forward windows; FP32 centre velocities of the forward
  // region, forward trace positions of the tile; the velocity window
  __host__ __device__ static constexpr size_t smem(int n, int m) {
    return sizeof(uint2) * (W3X * W3Y + W1X * W1Y + W2X * W2Y) +
           sizeof(float2) * (W2X * W2Y + TX * TY + vel_x(n, m) * vel_y(n, m));
  }
};
// the wide tile for dye grids at least 2x the velocity grid and 64 texels wide
inline bool dye_wide_tile(int n, int m) { return m >= 64 && m >= 2 * n; }

// 8-byte asynchronous global -> shared copy (no register staging) and its wait
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
// 16-byte variant (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

struct Rgb {
  float r, g, b;
};
__device__ __forceinline__ Rgb rgb_of(uint2 u) {
  const float2 rg = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
  return {rg.x, rg.y, __low2float(*reinterpret_cast<const __half2*>(&u.y))};
}
// binary16 texel (r, g, b, alpha 1) of FP32 channels, as a texture store rounds them
__device__ __forceinline__ uint2 pack_rgb(const Rgb& c) { return pack_texel(c.r, c.g, c.b, 1.f); }

// on-chip W x WY window of binary16 source texels with an exact global fallback
// (coordinates are wrapped indices)
template <int W, int WY>
struct SmemTex {
  static constexpr int w = W, wy = WY;
  const uint2* sm;
  int ox, oy, m;   // window origin (wrapped), dye grid size
  const uint2* g;
  __device__ __forceinline__ Rgb operator()(int x, int y) const {
    const int rx = (x - ox) & (m - 1), ry = (y - oy) & (m - 1);
    if (rx < w && ry < wy) return rgb_of(sm[ry * w + rx]);
    return rgb_of(__ldg(g + (size_t)y * m + x));
  }
  // the 2x2 footprint in one window test (slots rx, rx+1 hold texels x0, x1 = x0+1 wrapped)
  __device__ __forceinline__ bool quad(const Footprint& f, Rgb (&c)[4]) const {
    const int rx = (f.x0 - ox) & (m - 1), ry = (f.y0 - oy) & (m - 1);
    if (rx + 1 < w && ry + 1 < wy) {
      const uint2* p = sm + ry * w + rx;
      c[0] = rgb_of(p[0]);
      c[1] = rgb_of(p[1]);
      c[2] = rgb_of(p[w]);
      c[3] = rgb_of(p[w + 1]);
      return true;
    }
    return false;
  }
};
struct SmemVel {
  const float2* sm;
  int ox, oy, w, wy, n;   // window origin, row length (x extent), y extent
  const float2* g;
  __device__ __forceinline__ float2 operator()(int x, int y) const {
    const int rx = (x - ox) & (n - 1), ry = (y - oy) & (n - 1);
    if (rx < w && ry < wy) return sm[ry * w + rx];
    return __ldg(g + (size_t)y * n + x);
  }
};

// bilinear velocity with one window test for the 2x2 cell footprint (same arithmetic as sample_vel)
__device__ __forceinline__ float2 sample_vel_win(const SmemVel& vf, float px, float py) {
  const int n = vf.n;
  const float nf = (float)n;
  const float gx = __fmaf_rn(px, nf, -0.5f), gy = __fmaf_rn(py, nf, -0.5f);   // px * nf exact
  const float bx = floorf(gx), by = floorf(gy);
  const float fx = __fsub_rn(gx, bx), fy = __fsub_rn(gy, by);
  const int ix = (int)bx, iy = (int)by;
  const int rx = (ix - vf.ox) & (n - 1), ry = (iy - vf.oy) & (n - 1);
  float2 v00, v10, v01, v11;
  if (rx + 1 < vf.w && ry + 1 < vf.wy) {
    const float2* p = vf.sm + ry * vf.w + rx;
    v00 = p[0];
    v10 = p[1];
    v01 = p[vf.w];
    v11 = p[vf.w + 1];
  } else {
    const int x0 = ix & (n - 1), x1 = (ix + 1) & (n - 1), y0 = iy & (n - 1), y1 = (iy + 1) & (n - 1);
    v00 = vf(x0, y0);
    v10 = vf(x1, y0);
    v01 = vf(x0, y1);
    v11 = vf(x1, y1);
  }
  return lerp2v(lerp2v(v00, v10, fx), lerp2v(v01, v11, fx), fy);
}
struct WinVel {      // adapter: the window sampler where trace_from expects sample_vel
  const SmemVel& v;
};
__device__ __forceinline__ float2 sample_vel(const WinVel& w, float px, float py, int) {
  return sample_vel_win(w.v, px, py);
}

// r, g, b of the bilinear sample over a footprint, optionally with the 4-texel min / max
// (the same per-channel arithmetic as bilerp)
__device__ __forceinline__ Rgb bilerp_quad(const Rgb (&q)[4], const Footprint& f, Rgb* lo, Rgb* hi) {
  const Rgb c00 = q[0], c10 = q[1], c01 = q[2], c11 = q[3];
  if (lo) {
    lo->r = fminf(fminf(c00.r, c10.r), fminf(c01.r, c11.r));
    lo->g = fminf(fminf(c00.g, c10.g), fminf(c01.g, c11.g));
    lo->b = fminf(fminf(c00.b, c10.b), fminf(c01.b, c11.b));
    hi->r = fmaxf(fmaxf(c00.r, c10.r), fmaxf(c01.r, c11.r));
    hi->g = fmaxf(fmaxf(c00.g, c10.g), fmaxf(c01.g, c11.g));
    hi->b = fmaxf(fmaxf(c00.b, c10.b), fmaxf(c01.b, c11.b));
  }
  const float2 rg = lerp2v(lerp2v(make_float2(c00.r, c00.g), make_float2(c10.r, c10.g), f.fx),
                           lerp2v(make_float2(c01.r, c01.g), make_float2(c11.r, c11.g), f.fx), f.fy);
  return {rg.x, rg.y, lerp2(c00.b, c10.b, c01.b, c11.b, f.fx, f.fy)};
}
template <class TF>
__device__ __forceinline__ Rgb bilerp_rgb(const TF& tf, const Footprint& f, Rgb* lo = nullptr, Rgb* hi = nullptr) {
  Rgb q[4];
  if (!tf.quad(f, q)) {
    q[0] = tf(f.x0, f.y0);
    q[1] = tf(f.x1, f.y0);
    q[2] = tf(f.x0, f.y1);
    q[3] = tf(f.x1, f.y1);
  }
  return bilerp_quad(q, f, lo, hi);
}

// Window lookups without a bounds test, for a tile whose every trace moves less than one
// texel: each footprint then lies inside its window by construction of the halos, and the
// lookup reads the same slots (and does the same arithmetic) as the tested one above.
// Footprint of a sample for window lookups: the unwrapped texel of its lower corner and
// the weights (the arithmetic of footprint(); a window wraps the corner once, since
// ((x & (m-1)) - o) & (m-1) is (x - o) & (m-1) for a power-of-two m)
struct WinFoot {
  int ix, iy;
  float fx, fy;
};
__device__ __forceinline__ WinFoot win_foot(float sx, float sy, int m) {
  const float mf = (float)m;
  const float gx = __fmaf_rn(sx, mf, -0.5f), gy = __fmaf_rn(sy, mf, -0.5f);   // sx * mf exact
  const float bx = floorf(gx), by = floorf(gy);
  return {(int)bx, (int)by, __fsub_rn(gx, bx), __fsub_rn(gy, by)};
}
struct FastTex {   // binary16 window of row length W at wrapped origin (ox, oy)
  const uint2* sm;
  int w, ox, oy, m;
  __device__ __forceinline__ const uint2* at(const WinFoot& f) const {
    return sm + ((f.iy - oy) & (m - 1)) * w + ((f.ix - ox) & (m - 1));
  }
  __device__ __forceinline__ Rgb sample(const WinFoot& f, Rgb* lo = nullptr, Rgb* hi = nullptr) const {
    const uint2* p = at(f);
    const Rgb q[4] = {rgb_of(p[0]), rgb_of(p[1]), rgb_of(p[w]), rgb_of(p[w + 1])};
    Footprint fp;
    fp.fx = f.fx;
    fp.fy = f.fy;
    return bilerp_quad(q, fp, lo, hi);
  }
};
// the corrected pass's two samples over one footprint: a from the source window (with
// the 4-texel min / max), b from the backward window; r, g of each on the packed pipe as
// in bilerp_quad, and the two b channels together in one packed chain (each lane the
// arithmetic of lerp2)
__device__ __forceinline__ void sample_corr(const FastTex& ta, const FastTex& tb, const WinFoot& f, Rgb& a, Rgb& b,
                                            Rgb& lo, Rgb& hi) {
  const uint2* pa = ta.at(f);
  const uint2* pb = tb.at(f);
  const Rgb a00 = rgb_of(pa[0]), a10 = rgb_of(pa[1]), a01 = rgb_of(pa[ta.w]), a11 = rgb_of(pa[ta.w + 1]);
  const Rgb b00 = rgb_of(pb[0]), b10 = rgb_of(pb[1]), b01 = rgb_of(pb[tb.w]), b11 = rgb_of(pb[tb.w + 1]);
  lo.r = fminf(fminf(a00.r, a10.r), fminf(a01.r, a11.r));
  lo.g = fminf(fminf(a00.g, a10.g), fminf(a01.g, a11.g));
  lo.b = fminf(fminf(a00.b, a10.b), fminf(a01.b, a11.b));
  hi.r = fmaxf(fmaxf(a00.r, a10.r), fmaxf(a01.r, a11.r));
  hi.g = fmaxf(fmaxf(a00.g, a10.g), fmaxf(a01.g, a11.g));
  hi.b = fmaxf(fmaxf(a00.b, a10.b), fmaxf(a01.b, a11.b));
  const float2 arg = lerp2v(lerp2v(make_float2(a00.r, a00.g), make_float2(a10.r, a10.g), f.fx),
                            lerp2v(make_float2(a01.r, a01.g), make_float2(a11.r, a11.g), f.fx), f.fy);
  const float2 brg = lerp2v(lerp2v(make_float2(b00.r, b00.g), make_float2(b10.r, b10.g), f.fx),
                            lerp2v(make_float2(b01.r, b01.g), make_float2(b11.r, b11.g), f.fx), f.fy);
  const float2 bb = lerp2v(lerp2v(make_float2(a00.b, b00.b), make_float2(a10.b, b10.b), f.fx),
                           lerp2v(make_float2(a01.b, b01.b), make_float2(a11.b, b11.b), f.fx), f.fy);
  a = {arg.x, arg.y, bb.x};
  b = {brg.x, brg.y, bb.y};
}
struct FastVel {   // FP32 velocity window
  const float2* sm;
  int w, ox, oy, n;
};
__device__ __forceinline__ float2 sample_vel(const FastVel& v, float px, float py, int) {
  const int n = v.n;
  const float nf = (float)n;
  const float gx = __fmaf_rn(px, nf, -0.5f), gy = __fmaf_rn(py, nf, -0.5f);   // px * nf exact
  const float bx = floorf(gx), by = floorf(gy);
  const float fx = __fsub_rn(gx, bx), fy = __fsub_rn(gy, by);
  const float2* p = v.sm + (((int)by - v.oy) & (n - 1)) * v.w + (((int)bx - v.ox) & (n - 1));
  return lerp2v(lerp2v(p[0], p[1], fx), lerp2v(p[v.w], p[v.w + 1], fx), fy);
}
// velocity at the centre of dye texel (x, y) (wrapped indices) on a dye grid s = m / n
// times the velocity grid: the centre's velocity coordinate (2x + 1 - s) / (2s) is exact in
// FP32, so its floor and fraction -- the cell and the weight sample_vel derives from the
// position -- follow from integer arithmetic (lg2s = log2(2s), inv2s = 1/(2s)), and the
// lerps see the same operands
__device__ __forceinline__ float2 vel_centre(const FastVel& v, int x, int y, int s, int lg2s, float inv2s) {
  const int tx = 2 * x + 1 - s, ty = 2 * y + 1 - s;
  const float fx = (float)(tx & (2 * s - 1)) * inv2s, fy = (float)(ty & (2 * s - 1)) * inv2s;
  const int n = v.n;
  const float2* p = v.sm + (((ty >> lg2s) - v.oy) & (n - 1)) * v.w + (((tx >> lg2s) - v.ox) & (n - 1));
  return lerp2v(lerp2v(p[0], p[1], fx), lerp2v(p[v.w], p[v.w + 1], fx), fy);
}

// binary16 W x WY window whose texels outside the window are re-derived by EVAL
template <class EVAL, int W, int WY>
struct DerivedTex {
  static constexpr int w = W, wy = WY;
  const uint2* sm;
  int ox, oy, m;   // window origin (wrapped), dye grid size
  const EVAL& eval;
  __device__ __forceinline__ Rgb operator()(int x, int y) const {
    const int rx = (x - ox) & (m - 1), ry = (y - oy) & (m - 1);
    if (rx < w && ry < wy) return rgb_of(sm[ry * w + rx]);
    return rgb_of(eval(x, y));
  }
  __device__ __forceinline__ bool quad(const Footprint& f, Rgb (&c)[4]) const {
    const int rx = (f.x0 - ox) & (m - 1), ry = (f.y0 - oy) & (m - 1);
    if (rx + 1 < w && ry + 1 < wy) {
      const uint2* p = sm + ry * w + rx;
      c[0] = rgb_of(p[0]);
      c[1] = rgb_of(p[1]);
      c[2] = rgb_of(p[w]);
      c[3] = rgb_of(p[w + 1]);
      return true;
    }
    return false;
  }
};

// forward-pass texel (x, y) as the advect_fwd texture would hold it
template <class TS>
struct FwdEval {
  const SmemVel& vel;
  const TS& src;
  float h;
  int n, m;
  __device__ __forceinline__ uint2 operator()(int x, int y) const {
    const float2 p = texel_pos(x, y, m);
    const float2 s = trace_from(WinVel{vel}, p.x, p.y, sample_vel_win(vel, p.x, p.y), h, n);
    return pack_rgb(bilerp_rgb(src, footprint(s.x, s.y, m)));
  }
};
// backward-pass texel (x, y) as the advect_back texture would hold it
template <class FF>
struct BackEval {
  const SmemVel& vel;
  const FF& fwd;
  float h;
  int n, m;
  __device__ __forceinline__ uint2 operator()(int x, int y) const {
    const float2 p = texel_pos(x, y, m);
    const float2 s = trace_from(WinVel{vel}, p.x, p.y, sample_vel_win(vel, p.x, p.y), -h, n);
    return pack_rgb(bilerp_rgb(fwd, footprint(s.x, s.y, m)));
  }
};

// BFECC correction from r, g, b (the arithmetic of correct_from; alpha is not read)
template <class POS>
__device__ __forceinline__ uint2 correct_rgb(const Rgb& a, const Rgb& b, const Rgb& lo, const Rgb& hi, const POS& pos,
                                             float fade, const DevSplats* __restrict__ S) {
  const Rgba a4{a.r, a.g, a.b, 1.f}, b4{b.r, b.g, b.b, 1.f}, lo4{lo.r, lo.g, lo.b, 0.f}, hi4{hi.r, hi.g, hi.b, 0.f};
  return correct_from(a4, b4, lo4, hi4, pos, fade, S);
}

// Windows, origins and constants of one CTA of the fused dye kernel.
template <int TX> struct DyeCta {
  const float2* vel;
  const uint2* src;
  uint2* dst;
  const DevSplats* S;
  uint2 *s_src, *s_back, *s_fwd;
  float2 *s_v1, *s_sp, *s_vel;
  int n, m, tx0, ty0;
  int sx0, sy0, fx0, fy0, bx0, by0;   // wrapped origins of the source / forward / backward windows
  int vxw, vyw, vwx, vwy;             // velocity window: wrapped origin and extent
  float h, fade;
};

// The forward, backward and corrected passes of one tile.  FAST: every trace of the tile
// moves less than one texel (checked on the velocity window the traces read), so every
// footprint lies inside its window and the lookups skip the bounds tests and the
// recomputation from global memory; the arithmetic, and so the bits, are the same.
template <int TX, bool FAST>
__device__ __forceinline__ void dye_cta_passes(const DyeCta<TX>& c) {
  using G = DyeGeom<TX>;
  constexpr int TY = G::TY, NT = G::THREADS;
  constexpr int W1X = G::W1X, W1Y = G::W1Y, W2X = G::W2X, W2Y = G::W2Y, W3X = G::W3X, W3Y = G::W3Y;
  const int tid = threadIdx.x;
  const int n = c.n, m = c.m;
  const float h = c.h;
  const float inv_m = __frcp_rn((float)m);
  const int s = m / n, lg2s = 31 - __clz(2 * s);
  const float inv2s = __frcp_rn((float)(2 * s));
  const SmemVel V{c.s_vel, c.vxw, c.vyw, c.vwx, c.vwy, n, c.vel};
  const FastVel FV{c.s_vel, c.vwx, c.vxw, c.vyw, n};
  // velocity at the centre of texel (x, y), at position p
  auto vel_at = [&](int x, int y, float2 p) {
    if constexpr (FAST) return vel_centre(FV, x, y, s, lg2s, inv2s);
    else return sample_vel_win(V, p.x, p.y);
  };
  auto trace = [&](float px, float py, float2 v1, float hs) {
    if constexpr (FAST) return trace_from(FV, px, py, v1, hs, n);
    else return trace_from(WinVel{V}, px, py, v1, hs, n);
  };
  using Tex = SmemTex<W3X, W3Y>;
  const Tex T{c.s_src, c.sx0, c.sy0, m, c.src};
  const FastTex FT{c.s_src, W3X, c.sx0, c.sy0, m};

  // forward pass over the forward region (the source window is complete: the caller
  // waited for its copies before its barrier): the velocity at each texel centre (kept
  // for the -h trace), the forward trace from it -- kept for the tile's own texels, whose
  // corrected samples use it -- and the forward-pass texel it samples
  for (int i = tid; i < W2X * W2Y; i += NT) {
    const int ry = i / W2X, rx = i - ry * W2X;
    const int x = (c.fx0 + rx) & (m - 1), y = (c.fy0 + ry) & (m - 1);
    const float2 p = texel_pos(x, y, inv_m);
    const float2 v1 = vel_at(x, y, p);
    c.s_v1[i] = v1;
    const float2 sp = trace(p.x, p.y, v1, h);
    const int ix = rx - 2 * kDyeLo, iy = ry - 2 * kDyeLo;
    if ((unsigned)ix < (unsigned)TX && (unsigned)iy < (unsigned)TY) c.s_sp[iy * TX + ix] = sp;
    Rgb r;
    if constexpr (FAST) r = FT.sample(win_foot(sp.x, sp.y, m));
    else r = bilerp_rgb(T, footprint(sp.x, sp.y, m));
    c.s_fwd[i] = pack_rgb(r);
  }
  __syncthreads();

  using FE = FwdEval<Tex>;
  using FF = DerivedTex<FE, W2X, W2Y>;
  const FE fe{V, T, h, n, m};
  const FF ff{c.s_fwd, c.fx0, c.fy0, m, fe};
  const FastTex FFT{c.s_fwd, W2X, c.fx0, c.fy0, m};
  // backward pass over the backward region (nested in the forward region by kDyeLo / kDyeHi)
  for (int i = tid; i < W1X * W1Y; i += NT) {
    const int ry = i / W1X, rx = i - ry * W1X;
    const int fi = (ry + kDyeLo) * W2X + rx + kDyeLo;
    const float2 p = texel_pos((c.bx0 + rx) & (m - 1), (c.by0 + ry) & (m - 1), inv_m);
    const float2 sb = trace(p.x, p.y, c.s_v1[fi], -h);
    Rgb r;
    if constexpr (FAST) r = FFT.sample(win_foot(sb.x, sb.y, m));
    else r = bilerp_rgb(ff, footprint(sb.x, sb.y, m));
    c.s_back[i] = pack_rgb(r);
  }
  __syncthreads();

  using BE = BackEval<FF>;
  const BE be{V, ff, h, n, m};
  const DerivedTex<BE, W1X, W1Y> bf{c.s_back, c.bx0, c.by0, m, be};
  const FastTex FB{c.s_back, W1X, c.bx0, c.by0, m};
  for (int i = tid; i < TX * TY; i += NT) {
    const int ry = i / TX, rx = i - ry * TX;
    const int x = c.tx0 + rx, y = c.ty0 + ry;
    const float2 sp = c.s_sp[i];
    Rgb lo, hi, a, b;
    if constexpr (FAST) {
      sample_corr(FT, FB, win_foot(sp.x, sp.y, m), a, b, lo, hi);
    } else {
      const Footprint f = footprint(sp.x, sp.y, m);
      a = bilerp_rgb(T, f, &lo, &hi);
      b = bilerp_rgb(bf, f);
    }
    c.dst[(size_t)y * m + x] = correct_rgb(a, b, lo, hi, [&] { return texel_pos(x, y, inv_m); }, c.fade, c.S);
  }
}
// the context of this CTA from the kernel arguments
template <int TX>
__device__ __forceinline__ DyeCta<TX> dye_cta_setup(const float2* __restrict__ vel, const uint2* __restrict__ src,
                                                    uint2* __restrict__ dst, const float* __restrict__ dtbuf,
                                                    const DevParams* __restrict__ params,
                                                    const DevSplats* __restrict__ S, int n, int m) {
  using G = DyeGeom<TX>;
  constexpr int TY = G::TY;
  constexpr int W1X = G::W1X, W1Y = G::W1Y, W2X = G::W2X, W2Y = G::W2Y, W3X = G::W3X, W3Y = G::W3Y;
  extern __shared__ __align__(16) uint2 dsm2[];
  DyeCta<TX> c;
  c.vel = vel;
  c.src = src;
  c.dst = dst;
  c.S = S;
  c.s_src = dsm2;
  c.s_back = c.s_src + W3X * W3Y;
  c.s_fwd = c.s_back + W1X * W1Y;
  c.s_v1 = reinterpret_cast<float2*>(c.s_fwd + W2X * W2Y);   // velocity at forward-region texels
  c.s_sp = c.s_v1 + W2X * W2Y;                                // forward trace positions of the tile
  c.s_vel = c.s_sp + TX * TY;
  c.n = n;
  c.m = m;
  c.vwx = G::vel_x(n, m);
  c.vwy = G::vel_y(n, m);
  c.tx0 = blockIdx.x * TX;
  c.ty0 = blockIdx.y * TY;
  c.h = __fdiv_rn(dtbuf[0], kTwoPiF);
  c.fade = params->dye_fade;
  // origins (wrapped) of the on-chip windows
  c.sx0 = (c.tx0 - 3 * kDyeLo - 1) & (m - 1);   // even: rows of 16-byte texel pairs
  c.sy0 = (c.ty0 - 3 * kDyeLo) & (m - 1);
  c.fx0 = (c.tx0 - 2 * kDyeLo) & (m - 1);
  c.fy0 = (c.ty0 - 2 * kDyeLo) & (m - 1);
  c.bx0 = (c.tx0 - kDyeLo) & (m - 1);
  c.by0 = (c.ty0 - kDyeLo) & (m - 1);
  const int vx0 = (int)floorf(((float)(c.tx0 - 2 * kDyeLo - 1) + 0.5f) * (float)n / (float)m - 0.5f) - 1;
  const int vy0 = (int)floorf(((float)(c.ty0 - 2 * kDyeLo - 1) + 0.5f) * (float)n / (float)m - 0.5f) - 1;
  c.vxw = vx0 & (n - 1);
  c.vyw = vy0 & (n - 1);
  return c;
}

// the general passes kept out of line, from the kernel arguments: the rarely taken path
// with its recomputation chains neither sets the register budget of the fast path nor
// makes it keep its context in memory
template <int TX>
__device__ __noinline__ void dye_cta_passes_general(const float2* vel, const uint2* src, uint2* dst,
                                                    const float* dtbuf, const DevParams* params,
                                                    const DevSplats* S, int n, int m) {
  dye_cta_passes<TX, false>(dye_cta_setup<TX>(vel, src, dst, dtbuf, params, S, n, m));
}

template <int TX>
__global__ void __launch_bounds__(DyeGeom<TX>::THREADS, DyeGeom<TX>::MINB)
    k_dye_fused(const float2* __restrict__ vel, const uint2* __restrict__ src, uint2* __restrict__ dst,
                const float* __restrict__ dtbuf, const DevParams* __restrict__ params,
                const DevSplats* __restrict__ S, int n, int m) {
  using G = DyeGeom<TX>;
  constexpr int NT = G::THREADS, W3X = G::W3X, W3Y = G::W3Y;
  const DyeCta<TX> c = dye_cta_setup<TX>(vel, src, dst, dtbuf, params, S, n, m);
  const int tid = threadIdx.x;

  // the source window arrives asynchronously while the velocity window loads: one
  // warp per row, a texel pair per 16-byte copy (a pair starts on an even texel, so it
  // never straddles the periodic seam)
  const int warp = tid >> 5, lane = tid & 31;
  for (int ry = warp; ry < W3Y; ry += NT / 32) {
    const uint2* grow = src + (size_t)((c.sy0 + ry) & (m - 1)) * m;
    for (int k = lane; k < W3X / 2; k += 32) cp_async16(c.s_src + ry * W3X + 2 * k, grow + ((c.sx0 + 2 * k) & (m - 1)));
  }
  cp_async_commit();
  // the velocity window, and whether any of its values moves a trace a texel or more: a
  // sample's velocity is a convex combination of window values, so |u| h m < 0.99 and
  // |v| h m < 0.99 over the window bound every displacement of the tile below one texel
  const float lim = 0.99f / (fabsf(c.h) * (float)m);
  bool far = false;
  for (int ry = warp; ry < c.vwy; ry += NT / 32) {
    const float2* grow = vel + (size_t)((c.vyw + ry) & (n - 1)) * n;
    for (int rx = lane; rx < c.vwx; rx += 32) {
      const float2 v = __ldg(grow + ((c.vxw + rx) & (n - 1)));
      c.s_vel[ry * c.vwx + rx] = v;
      far |= !(fabsf(v.x) < lim && fabsf(v.y) < lim);
    }
  }
  // this thread's source copies have landed; the barrier below makes every thread's visible
  cp_async_wait_all();
  if (__syncthreads_or(far ? 1 : 0)) dye_cta_passes_general<TX>(vel, src, dst, dtbuf, params, S, n, m);
  else dye_cta_passes<TX, true>(c);
}

}  // namespace s2d
