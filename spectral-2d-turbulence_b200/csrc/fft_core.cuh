// fft_core.cuh -- register-blocked, shared-memory Stockham line FFT for sm_100a.
//
// A length-N line is spread over T = N/V threads; thread t holds the V elements
// t + T*m (m = 0..V-1) in registers ("natural distributed layout"), which is
// also the layout the transform leaves its result in.  The transform runs as
// P = ceil(log N / log V) Stockham autosort passes (Govindaraju et al., SC08):
// pass p does radix-R_p butterflies entirely in registers on elements N/R_p
// apart, twiddled by W_{Ns R}^{(j mod Ns) r}, and exchanges through a padded
// shared-memory line between passes.  The first pass reads registers loaded
// straight from HBM (coalesced, stride-T elements), the last pass leaves the
// outputs in registers for the caller's fused epilogue -- so a whole-line
// transform costs P-1 shared-memory round trips and no global ping-pong.
//
// The reference kernel (fft.wgsl:42-79) is an in-place radix-4 DIT with a
// digit-reversal scatter on load and one smem round trip per radix-4 stage;
// here the exchange between two radix-V passes IS the base-V digit transposition
// (for P = 2 it is exactly the digit reversal of fft_ref.py:19-24 over [V, V]),
// so the permutation is folded into the exchange instead of a separate scatter.
#pragma once
#include <cuda_runtime.h>
#include <utility>

namespace s2d {

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

// cos(2*pi*k/64), quarter-wave table (double literals, rounded once to float)
__host__ __device__ constexpr double cos64_q(int k) {
  return k == 0 ? 1.0 : k == 1 ? 0.99518472667219693 : k == 2 ? 0.98078528040323043
       : k == 3 ? 0.95694033573220882 : k == 4 ? 0.92387953251128674 : k == 5 ? 0.88192126434835505
       : k == 6 ? 0.83146961230254524 : k == 7 ? 0.77301045336273699 : k == 8 ? 0.70710678118654757
       : k == 9 ? 0.63439328416364549 : k == 10 ? 0.55557023301960229 : k == 11 ? 0.47139673682599781
       : k == 12 ? 0.38268343236508984 : k == 13 ? 0.29028467725446233 : k == 14 ? 0.19509032201612833
       : k == 15 ? 0.09801714032956077 : 0.0;
}
__host__ __device__ constexpr double cos64(int k) {
  k &= 63;
  return k <= 16 ? cos64_q(k) : k <= 32 ? -cos64_q(32 - k) : k <= 48 ? -cos64_q(k - 32) : cos64_q(64 - k);
}
__host__ __device__ constexpr double sin64(int k) { return cos64(k - 16); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by SIGN*i
template <int SIGN> __device__ __forceinline__ float2 cmul_si(float2 a) {
  return SIGN > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// a * W_R^E with W_R = exp(SIGN * 2*pi*i / R), R | 64, E compile-time after unrolling
template <int SIGN, int R>
__device__ __forceinline__ float2 twmul_c(float2 a, int e) {
  const int k = ((e % R) + R) % R * (64 / R);
  if (k == 0) return a;
  if (k == 16) return cmul_si<SIGN>(a);
  if (k == 32) return make_float2(-a.x, -a.y);
  if (k == 48) return cmul_si<-SIGN>(a);
  const float c = (float)cos64(k), s = (float)(SIGN * sin64(k));
  return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
}

// ------------------------------------------------------------------ in-register DFTs
// Natural order in and out: v[k] <- sum_n v[n] W_R^{nk}, W_R = exp(SIGN 2 pi i / R).
template <int R, int SIGN> struct Dft;

template <int SIGN> struct Dft<1, SIGN> {
  __device__ __forceinline__ static void run(float2*) {}
};
template <int SIGN> struct Dft<2, SIGN> {
  __device__ __forceinline__ static void run(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <int SIGN> struct Dft<4, SIGN> {
  __device__ __forceinline__ static void run(float2* v) {
    float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    float2 s13 = cadd(v[1], v[3]), d13 = cmul_si<SIGN>(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[1] = cadd(d02, d13);
    v[2] = csub(s02, s13);
    v[3] = csub(d02, d13);
  }
};
// R = P*Q, n = Q*n1 + n2, k = k1 + P*k2 (four-step inside registers)
template <int R, int SIGN> struct Dft {
  static constexpr int P = (R % 4 == 0 && R / 4 >= 2) ? 4 : 2;
  static constexpr int Q = R / P;
  __device__ __forceinline__ static void run(float2* v) {
    float2 y[Q][P];
#pragma unroll
    for (int n2 = 0; n2 < Q; ++n2) {
      float2 t[P];
#pragma unroll
      for (int n1 = 0; n1 < P; ++n1) t[n1] = v[Q * n1 + n2];
      Dft<P, SIGN>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) y[n2][k1] = twmul_c<SIGN, R>(t[k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      float2 t[Q];
#pragma unroll
      for (int n2 = 0; n2 < Q; ++n2) t[n2] = y[n2][k1];
      Dft<Q, SIGN>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < Q; ++k2) v[k1 + P * k2] = t[k2];
    }
  }
};

// ------------------------------------------------------------------ line plans
template <int N_, int V_> struct LinePlan {
  static constexpr int N = N_, V = V_, T = N / V;
  static constexpr int LOGN = ilog2c(N), LOGV = ilog2c(V);
  static constexpr int P = (LOGN + LOGV - 1) / LOGV;
  __host__ __device__ static constexpr int radix(int p) { return p < P - 1 ? V : (N >> (LOGV * (P - 1))); }
  __host__ __device__ static constexpr int ns(int p) { return 1 << (LOGV * p); }
  // padded shared-memory index: one pad slot every 16 elements keeps the
  // stride-R stores of the first pass free of bank conflicts
  __host__ __device__ static constexpr int pad(int i) { return i + (i >> 4); }
  static constexpr int PADDED = N + N / 16;
  // line stride in float2 with a chosen residue mod 16 (bank offset between lines)
  __host__ __device__ static constexpr int stride(int residue) {
    return PADDED + (((residue - PADDED) % 16) + 16) % 16;
  }
  static_assert(N >= V, "line shorter than the per-thread block");
  static_assert((N & (N - 1)) == 0, "power-of-two lines only");
};

template <int I> using ic = std::integral_constant<int, I>;
template <class F, int... I>
__device__ __forceinline__ void sfor_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(ic<I>{}), ...);
}
template <int N, class F> __device__ __forceinline__ void sfor(F&& f) {
  sfor_impl(f, std::make_integer_sequence<int, N>{});
}

// Twiddle W_N^e for the pass twiddles, from an FP64-generated table of
// exp(-2 pi i m / N), m < N (forward sign); the inverse uses the conjugate.
template <int SIGN> __device__ __forceinline__ float2 table_tw(const float2* __restrict__ tw, int e) {
  float2 w = __ldg(tw + e);
  return SIGN < 0 ? w : make_float2(w.x, -w.y);
}

// K lines transformed in lockstep (their exchanges share barriers).
//   x[q][m]  : element t + T*m of line q, in and out (natural distributed layout)
//   buf[q]   : padded smem line of line q (PADDED float2 at least)
//   sync()   : barrier over every thread that shares the buffers
template <int N, int V, int SIGN, int K, class Sync>
__device__ __forceinline__ void fft_lines(float2 (&x)[K][V], float2* const (&buf)[K], int t,
                                          const float2* __restrict__ tw, Sync&& sync) {
  using PL = LinePlan<N, V>;
  constexpr int T = PL::T;
  sfor<PL::P>([&](auto pc) {
    constexpr int p = decltype(pc)::value;
    constexpr int R = PL::radix(p), B = V / R, NS = PL::ns(p);
    float2 v[K][V];
    if constexpr (p == 0) {
#pragma unroll
      for (int q = 0; q < K; ++q)
#pragma unroll
        for (int b = 0; b < B; ++b)
#pragma unroll
          for (int r = 0; r < R; ++r) v[q][b * R + r] = x[q][b + B * r];
    } else {
#pragma unroll
      for (int q = 0; q < K; ++q)
#pragma unroll
        for (int b = 0; b < B; ++b) {
          const int j = t + T * b;
#pragma unroll
          for (int r = 0; r < R; ++r) v[q][b * R + r] = buf[q][PL::pad(j + r * (N / R))];
        }
      sync();
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int j = t + T * b;
        const int jm = j & (NS - 1);
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const float2 w = table_tw<SIGN>(tw, jm * r * (N / (NS * R)));
#pragma unroll
          for (int q = 0; q < K; ++q) v[q][b * R + r] = cmul(v[q][b * R + r], w);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < K; ++q)
#pragma unroll
      for (int b = 0; b < B; ++b) Dft<R, SIGN>::run(&v[q][b * R]);
    if constexpr (p < PL::P - 1) {
#pragma unroll
      for (int q = 0; q < K; ++q)
#pragma unroll
        for (int b = 0; b < B; ++b) {
          const int j = t + T * b;
          const int base = (j / NS) * NS * R + (j & (NS - 1));
#pragma unroll
          for (int r = 0; r < R; ++r) buf[q][PL::pad(base + r * NS)] = v[q][b * R + r];
        }
      sync();
    } else {
#pragma unroll
      for (int q = 0; q < K; ++q)
#pragma unroll
        for (int b = 0; b < B; ++b)
#pragma unroll
          for (int r = 0; r < R; ++r) x[q][b + B * r] = v[q][b * R + r];
    }
  });
}

}  // namespace s2d
