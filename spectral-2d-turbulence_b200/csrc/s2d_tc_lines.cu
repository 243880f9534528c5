// s2d_tc_lines.cu -- tensor-core line transforms of N = N1 x N2 points for the grid sizes
// other than 1024 (256 = 16 x 16, 512 = 32 x 16, 2048 = 32 x 64, 4096 = 64 x 64).
//
// The four-step form of s2d_tc.cuh with general factors: x[n1 + N1 n2] --(DFT_N2 over n2,
// a GEMM)--> Y[n1][k2], Y *= W_N^{n1 k2} (FP32, CUDA cores), --(DFT_N1 over n1, a GEMM)-->
// X[k2 + N2 k1].  Each DFT_R is the real block form of the R-point matrix (K = N = 2R
// halves) applied as split hi + lo FP16 / BF16 products accumulated in FP32 in tensor
// memory; the inverse is conj(F(conj x)), so only forward matrices and twiddles exist.
//
// One warpgroup (128 threads) per CTA transforms L lines, L = max(128 / N1, 128 / N2), so
// that both GEMMs are whole M = 128 blocks (BA = N1 L / 128 and BC = N2 L / 128 of them).
// Step-A rows carry their own power-of-two scale; step-C rows take the CTA bound
// N2 max|x| (|Y| <= sum |x|).  Rows (n1, line) are ordered n1-fastest for a row pass
// (AXIS 0: a warp's loads are consecutive in x) and line-fastest for a column pass.
//
// These transforms serve the tensor-core solvers at those sizes, whose step runs the
// reference's unfused stage order (velocity pack, inverse transforms, products, forward
// transform, assemble, RK3 update); the fused tensor-core stages exist at 1024^2.
#include <cuda_runtime.h>

#include <type_traits>

#include "s2d_tc.cuh"
#include "s2d_tc_lines.h"

namespace s2d {
namespace tc {
namespace {

// K-major, no-swizzle operand of K halves per row: core matrices 8 rows x 16 bytes,
// K-adjacent 128 bytes apart (LBO), 8-row groups 16 K bytes apart (SBO)
__device__ __forceinline__ uint32_t g_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (16 * K) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
// bytes of one plane of the real block DFT_R matrix (2R rows x 2R halves)
__host__ __device__ constexpr int dft_plane_bytes(int R) { return 8 * R * R; }

// DFT_R, forward sign, W_R^{nk} = W_N^{(N/R) n k} from the FP64-generated table
// tw[m] = exp(-2 pi i m / N): row 2k holds (c, -s) and row 2k+1 (s, c) at K = 2n, 2n+1
template <class P>
__global__ void k_dft_block(char* out, int R, const float2* __restrict__ tw, int N) {
  const int K = 2 * R;
  char* hi = out;
  char* lo = out + dft_plane_bytes(R);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < R * R; e += gridDim.x * blockDim.x) {
    const int k = e / R, n = e - (e / R) * R;
    const float2 w = __ldg(tw + (int)(((long long)(N / R) * n * k) % N));
    const float c = w.x, s = w.y;
    typename P::H2 h, l;
    split2<P>(c, -s, h, l);
    uint32_t o = g_off(2 * k, 2 * n, K);
    *reinterpret_cast<typename P::H2*>(hi + o) = h;
    *reinterpret_cast<typename P::H2*>(lo + o) = l;
    split2<P>(s, c, h, l);
    o = g_off(2 * k + 1, 2 * n, K);
    *reinterpret_cast<typename P::H2*>(hi + o) = h;
    *reinterpret_cast<typename P::H2*>(lo + o) = l;
  }
}

template <int N1, int N2> struct LineGeom {
  static constexpr int N = N1 * N2;
  static constexpr int L = (128 / N1 > 128 / N2) ? 128 / N1 : 128 / N2;   // lines per CTA
  static constexpr int BA = N1 * L / 128, BC = N2 * L / 128;              // M = 128 blocks per GEMM
  static constexpr int KA = 2 * N2, KC = 2 * N1;                          // K (= N) of the two GEMMs
  static constexpr int OP = (BA * 128 * KA > BC * 128 * KC ? BA * 128 * KA : BC * 128 * KC) * 2;   // plane bytes
  static constexpr int TA = dft_plane_bytes(N2), TC = dft_plane_bytes(N1);
  static constexpr bool SAME = N1 == N2;
  static constexpr int OFF_OP = 0;
  static constexpr int OFF_TA = 2 * OP;
  static constexpr int OFF_TC = OFF_TA + 2 * TA;
  static constexpr int OFF_MISC = OFF_TC + (SAME ? 0 : 2 * TC);
  // at most 4 CTAs per SM (228 KB / 4), so their 128-column TMEM allocations fit the SM's 512
  // and tcgen05.alloc never waits for another CTA
  static constexpr int SMEM = OFF_MISC + 128 > 56 * 1024 ? OFF_MISC + 128 : 56 * 1024;
  static constexpr int TAB = 2 * TA + (SAME ? 0 : 2 * TC);   // global table bytes
  static_assert(BA * KA <= 128 && BC * KC <= 128, "accumulators fit 128 TMEM columns");
  static_assert(N2 * L % 128 == 0 && N1 * L % 128 == 0, "whole M = 128 blocks");
};

template <class P>
__device__ __forceinline__ void g_gemm3(uint32_t tmem_d, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi, uint32_t b_lo,
                                        int K) {
  const uint32_t idesc = idesc_f16(128, K, P::kFmt);
  for (int kb = 0; kb < K / 16; ++kb) {
    const uint32_t o = (uint32_t)kb * 256;
    const uint32_t sbo = 16u * (uint32_t)K;
    mma_f16(tmem_d, smem_desc(a_hi + o, 128, sbo), smem_desc(b_hi + o, 128, sbo), idesc, kb > 0 ? 1u : 0u);
    mma_f16(tmem_d, smem_desc(a_hi + o, 128, sbo), smem_desc(b_lo + o, 128, sbo), idesc, 1u);
    mma_f16(tmem_d, smem_desc(a_lo + o, 128, sbo), smem_desc(b_hi + o, 128, sbo), idesc, 1u);
  }
}

// One pass (AXIS 0 = rows, 1 = columns) of the 2D transform over L lines of an N x N
// field, in place.  Forward unscaled, inverse scaled 1/N per pass (fft.js:58-59).
template <int N1, int N2, int AXIS, int SIGN, class P>
__global__ void __launch_bounds__(128) k_fft_tcg(float2* data, const char* __restrict__ tab,
                                                 const float2* __restrict__ tw, int* err) {
  using G = LineGeom<N1, N2>;
  constexpr int N = G::N, L = G::L, KA = G::KA, KC = G::KC;
  extern __shared__ __align__(1024) char sm[];
  char* op_hi = sm + G::OFF_OP;
  char* op_lo = op_hi + G::OP;
  uint64_t* setup = reinterpret_cast<uint64_t*>(sm + G::OFF_MISC);
  uint64_t* bar = setup + 1;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + G::OFF_MISC + 16);
  float* wmax = reinterpret_cast<float*>(sm + G::OFF_MISC + 32);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int l0 = blockIdx.x * L;
  const uint32_t s_op_hi = smem_u32(op_hi), s_op_lo = smem_u32(op_lo);
  const uint32_t s_ta = smem_u32(sm + G::OFF_TA), s_tc = smem_u32(sm + (G::SAME ? G::OFF_TA : G::OFF_TC));
  const int tcb = G::SAME ? G::TA : G::TC;   // plane bytes of the step-C matrix

  if (warp == 0) {
    tmem_alloc(tslot, 128);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(setup, 1);
    mbar_init(bar, 1);
    mbar_fence_init();
    mbar_arrive_expect_tx(setup, (uint32_t)G::TAB);
    bulk_g2s(sm + G::OFF_TA, tab, (uint32_t)G::TAB, setup);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
  auto elem = [&](int line, int n) -> float2* {
    return AXIS == 0 ? data + (size_t)(l0 + line) * N + n : data + (size_t)n * N + l0 + line;
  };

  // ---- step A operand: rows r = b * 128 + tid, (n1, line); per-row scale, conj for the inverse
  float sA[G::BA];
  float mx_all = 0.f;
#pragma unroll
  for (int b = 0; b < G::BA; ++b) {
    const int r = b * 128 + tid;
    const int n1 = AXIS == 0 ? r % N1 : r / L, line = AXIS == 0 ? r / N1 : r % L;
    float mx = 0.f;
    for (int n2 = 0; n2 < N2; ++n2) {
      const float2 v = *elem(line, n1 + N1 * n2);
      mx = fmaxf(mx, fmaxf(fabsf(v.x), fabsf(v.y)));
    }
    sA[b] = pow2_scale(mx);
    mx_all = fmaxf(mx_all, mx);
    const float si = SIGN > 0 ? -sA[b] : sA[b];
    for (int n2 = 0; n2 < N2; ++n2) {
      const float2 v = *elem(line, n1 + N1 * n2);
      typename P::H2 h, l;
      split2<P>(v.x * sA[b], v.y * si, h, l);
      const uint32_t o = g_off(r, 2 * n2, KA);
      *reinterpret_cast<typename P::H2*>(op_hi + o) = h;
      *reinterpret_cast<typename P::H2*>(op_lo + o) = l;
    }
  }
  mx_all = warp_max(mx_all);
  if (lane == 0) wmax[warp] = mx_all;
  fence_proxy_async();
  fence_before_sync();
  __syncthreads();
  if (tid == 0) {
    mbar_wait_bounded(setup, 0u, err, 4);
    fence_after_sync();
#pragma unroll
    for (int b = 0; b < G::BA; ++b)
      g_gemm3<P>(tmem + (uint32_t)(b * KA), s_op_hi + (uint32_t)(b * 128 * KA * 2), s_op_lo + (uint32_t)(b * 128 * KA * 2),
                 s_ta, s_ta + (uint32_t)G::TA, KA);
    mma_commit(bar);
  }
  const float mall = fmaxf(fmaxf(wmax[0], wmax[1]), fmaxf(wmax[2], wmax[3]));
  const float sC = pow2_scale(mall * (float)N2);
  bool bad = !mbar_wait_bounded(bar, 0u, err, 2);
  fence_after_sync();
  // ---- step A done: row (n1, line) holds Y[k2]; twiddle into the step-C operand rows
  // (k2, line) at K = n1 (the step-A operands are dead: their GEMMs have completed)
#pragma unroll
  for (int b = 0; b < G::BA; ++b) {
    const int r = b * 128 + tid;
    const int n1 = AXIS == 0 ? r % N1 : r / L, line = AXIS == 0 ? r / N1 : r % L;
    const float f = sC / sA[b];
    for (int c = 0; c < KA / 16; ++c) {
      float y[16];
      tmem_ld16(tmem + lane_off + (uint32_t)(b * KA + 16 * c), y);
      tmem_wait_ld();
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int k2 = 8 * c + e;
        const float2 w = __ldg(tw + n1 * k2);
        const float re = (y[2 * e] * w.x - y[2 * e + 1] * w.y) * f;
        const float im = (y[2 * e] * w.y + y[2 * e + 1] * w.x) * f;
        const int rc = AXIS == 0 ? line * N2 + k2 : k2 * L + line;
        typename P::H2 h, l;
        split2<P>(re, im, h, l);
        const uint32_t o = g_off(rc, 2 * n1, KC);
        *reinterpret_cast<typename P::H2*>(op_hi + o) = h;
        *reinterpret_cast<typename P::H2*>(op_lo + o) = l;
      }
    }
  }
  fence_proxy_async();
  fence_before_sync();
  const int gave_up = __syncthreads_or(bad ? 1 : 0);   // uniform: a wait gave up, issue nothing more
  if (tid == 0 && !gave_up) {
    fence_after_sync();
#pragma unroll
    for (int b = 0; b < G::BC; ++b)
      g_gemm3<P>(tmem + (uint32_t)(b * KC), s_op_hi + (uint32_t)(b * 128 * KC * 2), s_op_lo + (uint32_t)(b * 128 * KC * 2),
                 s_tc, s_tc + (uint32_t)tcb, KC);
    mma_commit(bar);
  }
  if (!gave_up) bad |= !mbar_wait_bounded(bar, 1u, err, 3);
  fence_after_sync();
  // ---- step C done: row (k2, line) holds X[k2 + N2 k1] (results invalid if a wait gave up)
  const float post = (SIGN > 0 ? 1.f / (float)N : 1.f) / sC;
#pragma unroll
  for (int b = 0; b < G::BC; ++b) {
    const int r = b * 128 + tid;
    const int k2 = AXIS == 0 ? r % N2 : r / L, line = AXIS == 0 ? r / N2 : r % L;
    for (int c = 0; c < KC / 16; ++c) {
      float y[16];
      tmem_ld16(tmem + lane_off + (uint32_t)(b * KC + 16 * c), y);
      tmem_wait_ld();
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int k1 = 8 * c + e;
        *elem(line, k2 + N2 * k1) = make_float2(y[2 * e] * post, (SIGN > 0 ? -y[2 * e + 1] : y[2 * e + 1]) * post);
      }
    }
  }
  fence_before_sync();
  if (__syncthreads_or(bad ? 1 : 0) && tid == 0) {
    // a GEMM or the table copy may still be in flight: wait for it (bounded) before the
    // TMEM and shared memory it writes are released
    mbar_wait_bounded(setup, 0u, nullptr, 0);
    mbar_wait_bounded(bar, gave_up ? 0u : 1u, nullptr, 0);
  }
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, 128);
  }
}

template <int N1, int N2, class P> cudaError_t attrs_for() {
  using G = LineGeom<N1, N2>;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) { if (r != cudaSuccess && e == cudaSuccess) e = r; };
  chk(cudaFuncSetAttribute(k_fft_tcg<N1, N2, 0, -1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
  chk(cudaFuncSetAttribute(k_fft_tcg<N1, N2, 0, +1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
  chk(cudaFuncSetAttribute(k_fft_tcg<N1, N2, 1, -1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
  chk(cudaFuncSetAttribute(k_fft_tcg<N1, N2, 1, +1, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
  return e;
}

template <int N1, int N2, class P>
void fft2_for(float2* buf, int sign, const char* tab, const float2* tw, int* err, cudaStream_t st) {
  using G = LineGeom<N1, N2>;
  const dim3 g(G::N / G::L), b(128);
  if (sign < 0) {
    k_fft_tcg<N1, N2, 0, -1, P><<<g, b, G::SMEM, st>>>(buf, tab, tw, err);
    k_fft_tcg<N1, N2, 1, -1, P><<<g, b, G::SMEM, st>>>(buf, tab, tw, err);
  } else {
    k_fft_tcg<N1, N2, 0, +1, P><<<g, b, G::SMEM, st>>>(buf, tab, tw, err);
    k_fft_tcg<N1, N2, 1, +1, P><<<g, b, G::SMEM, st>>>(buf, tab, tw, err);
  }
}

template <int N1, int N2, class P> void tables_for(char* tab, const float2* tw, cudaStream_t st) {
  using G = LineGeom<N1, N2>;
  k_dft_block<P><<<4, 256, 0, st>>>(tab, N2, tw, G::N);
  if (!G::SAME) k_dft_block<P><<<4, 256, 0, st>>>(tab + 2 * G::TA, N1, tw, G::N);
}

// factors of the supported sizes
template <class F> bool with_factors(int n, F&& f) {
  switch (n) {
    case 256: f(std::integral_constant<int, 16>{}, std::integral_constant<int, 16>{}); return true;
    case 512: f(std::integral_constant<int, 32>{}, std::integral_constant<int, 16>{}); return true;
    case 2048: f(std::integral_constant<int, 32>{}, std::integral_constant<int, 64>{}); return true;
    case 4096: f(std::integral_constant<int, 64>{}, std::integral_constant<int, 64>{}); return true;
    default: return false;
  }
}

}  // namespace

bool tc_lines_supported(int n) { return n == 256 || n == 512 || n == 2048 || n == 4096; }

size_t tc_lines_table_bytes(int n) {
  size_t out = 0;
  with_factors(n, [&](auto a, auto b) { out = (size_t)LineGeom<decltype(a)::value, decltype(b)::value>::TAB; });
  return out;
}

cudaError_t tc_lines_attrs(int n, int bf16) {
  cudaError_t e = cudaErrorInvalidValue;
  with_factors(n, [&](auto a, auto b) {
    constexpr int A = decltype(a)::value, B = decltype(b)::value;
    e = bf16 ? attrs_for<A, B, PrecBF16>() : attrs_for<A, B, PrecF16>();
  });
  return e;
}

void tc_lines_tables(int n, int bf16, char* tab, const float2* tw, cudaStream_t st) {
  with_factors(n, [&](auto a, auto b) {
    constexpr int A = decltype(a)::value, B = decltype(b)::value;
    if (bf16) tables_for<A, B, PrecBF16>(tab, tw, st);
    else tables_for<A, B, PrecF16>(tab, tw, st);
  });
}

void tc_lines_fft2(int n, int bf16, float2* buf, int sign, const char* tab, const float2* tw, int* err,
                   cudaStream_t st) {
  with_factors(n, [&](auto a, auto b) {
    constexpr int A = decltype(a)::value, B = decltype(b)::value;
    if (bf16) fft2_for<A, B, PrecBF16>(buf, sign, tab, tw, err, st);
    else fft2_for<A, B, PrecF16>(buf, sign, tab, tw, err, st);
  });
}

}  // namespace tc
}  // namespace s2d
