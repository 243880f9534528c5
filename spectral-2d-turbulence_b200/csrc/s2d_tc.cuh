// s2d_tc.cuh -- tensor-core (tcgen05) DFT-GEMM line transforms for sm_100a.
//
// A 1024-point line is transformed in the four-step form N = 32 x 32:
//   x[n1 + 32 n2] --(DFT32 over n2, a GEMM)--> Y[n1][k2]
//   Y *= W_1024^{n1 k2}                        (FP32 twiddle, CUDA cores)
//   Y --(DFT32 over n1, a GEMM)--> X[k2 + 32 k1]
// Each DFT32 is a real GEMM D[M x 64] = A[M x 64] . B[64 x 64]: rows of A are
// (line, fixed index) with the 32 complex inputs as 64 interleaved (re, im)
// values along K; B is the real block form of the 32 x 32 DFT matrix.
// Operands are FP16 split as hi + lo with x ~= hi + lo and the three products
// hi.hi + hi.lo + lo.hi accumulated in FP32 in tensor memory (TMEM); a per-CTA
// power-of-two scale keeps every operand inside FP16 range (scaling is exact).
//
// tcgen05 usage: one elected thread issues tcgen05.mma (cta_group::1,
// kind::f16, M = 128, N = 64, K = 16, A and B K-major in shared memory, no
// swizzle: 8 x 16-byte core matrices, LBO = 128 B between K-adjacent and
// SBO = 1024 B between M-adjacent core matrices), tcgen05.commit arrives on an
// mbarrier, and every warp reads its 32 TMEM lanes back with tcgen05.ld.
#pragma once
#include <cuda_fp16.h>
#include "s2d_async.cuh"
#include "s2d_device.cuh"
#include "s2d_kernels.cuh"

namespace s2d {
namespace tc {

// ------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {   // whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {                              // whole warp
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {   // whole warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns, lane i of the warp -> register set of thread i
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ------------------------------------------------------------------ descriptors
// shared-memory matrix descriptor, K-major, no swizzle (sm100 version 1)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// instruction descriptor: FP16 x FP16 -> FP32, A and B K-major, M x N
__host__ __device__ constexpr uint32_t idesc_f16(int m, int n) {
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// ------------------------------------------------------------------ operand layout
constexpr int kK = 64;                  // real K of a DFT32 (32 complex inputs)
constexpr uint32_t kLBO = 128;          // bytes between K-adjacent core matrices
constexpr uint32_t kSBO = 1024;         // bytes between M-adjacent 8-row groups (8 K chunks x 128 B)
constexpr int kBlockBytes = 128 * kK * 2;   // one M=128 block, one plane (16 KB)
constexpr int kBBytes = 64 * kK * 2;        // the 64 x 64 DFT matrix, one plane (8 KB)

// byte offset of element (row r, k) in a K-major no-swizzle operand of K = 64
__device__ __forceinline__ uint32_t op_off(int r, int k) {
  return (uint32_t)((r >> 3) * kSBO + (k >> 3) * kLBO + (r & 7) * 16 + (k & 7) * 2);
}

// split x into hi + lo (FP16) with x ~= hi + lo
__device__ __forceinline__ void split2(float re, float im, __half2& hi, __half2& lo) {
  hi = __floats2half2_rn(re, im);
  const float2 h = __half22float2(hi);
  lo = __floats2half2_rn(re - h.x, im - h.y);
}
// store complex (re, im) at row r, complex column j (K = 2j, 2j+1) of the hi and lo planes
__device__ __forceinline__ void put_c(char* hi_plane, char* lo_plane, int r, int j, float re, float im) {
  __half2 h, l;
  split2(re, im, h, l);
  const uint32_t o = op_off(r, 2 * j);
  *reinterpret_cast<__half2*>(hi_plane + o) = h;
  *reinterpret_cast<__half2*>(lo_plane + o) = l;
}

// Real block form of the 32-point DFT with sign SIGN, stored transposed (row = output
// real index n, K = input real index): for output k2 and input n2, W = c + i s,
//   Bt[2k2][2n2] = c, Bt[2k2][2n2+1] = -s, Bt[2k2+1][2n2] = s, Bt[2k2+1][2n2+1] = c.
// W_32^{n2 k2} = W_1024^{32 n2 k2} from the FP64-generated twiddle table (forward sign).
template <int SIGN>
__device__ __forceinline__ void build_dft32(char* hi_plane, char* lo_plane, const float2* __restrict__ tw1024) {
  for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
    const int k2 = e >> 5, n2 = e & 31;
    float2 w = __ldg(tw1024 + ((32 * n2 * k2) & 1023));
    if (SIGN > 0) w.y = -w.y;
    const float c = w.x, s = w.y;
    __half2 h, l;
    // row 2k2: (c, -s) at K = 2n2, 2n2+1
    split2(c, -s, h, l);
    uint32_t o = op_off(2 * k2, 2 * n2);
    *reinterpret_cast<__half2*>(hi_plane + o) = h;
    *reinterpret_cast<__half2*>(lo_plane + o) = l;
    // row 2k2+1: (s, c)
    split2(s, c, h, l);
    o = op_off(2 * k2 + 1, 2 * n2);
    *reinterpret_cast<__half2*>(hi_plane + o) = h;
    *reinterpret_cast<__half2*>(lo_plane + o) = l;
  }
}

// D(block b) = A(block b) . B over K = 64: hi.hi + hi.lo + lo.hi, 3 x 4 MMAs of K = 16
__device__ __forceinline__ void issue_dft_gemm(uint32_t tmem_d, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi,
                                               uint32_t b_lo) {
  constexpr uint32_t idesc = idesc_f16(128, 64);
  uint32_t acc = 0;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    const uint32_t ko = (uint32_t)kb * 2 * kLBO;   // two 8-element K chunks per MMA
    mma_f16(tmem_d, smem_desc(a_hi + ko, kLBO, kSBO), smem_desc(b_hi + ko, kLBO, kSBO), idesc, acc);
    acc = 1;
    mma_f16(tmem_d, smem_desc(a_hi + ko, kLBO, kSBO), smem_desc(b_lo + ko, kLBO, kSBO), idesc, 1);
    mma_f16(tmem_d, smem_desc(a_lo + ko, kLBO, kSBO), smem_desc(b_hi + ko, kLBO, kSBO), idesc, 1);
  }
}

// CTA-wide max of a non-negative float through a shared word (all threads call)
__device__ __forceinline__ float cta_max(float v, unsigned* word) {
  v = warp_max(v);
  if (threadIdx.x == 0) *word = 0u;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) atomicMax(word, __float_as_uint(v));
  __syncthreads();
  return __uint_as_float(*word);
}

// power-of-two scale that maps max |x| to at most 2^14 (FP16 max is 65504)
__device__ __forceinline__ float pow2_scale(float maxabs) {
  if (!(maxabs > 0.f) || !isfinite(maxabs)) return 1.f;
  const int e = ilogbf(maxabs);                       // maxabs in [2^e, 2^(e+1))
  return ldexpf(1.f, 13 - e);
}

}  // namespace tc
}  // namespace s2d

namespace s2d {
namespace tc {

// shared-memory plan of the 8-line transform CTA
constexpr int kTcLines = 8;                       // lines per CTA: two M = 128 blocks
constexpr int kTcThreads = 256;
constexpr int kTcAHi = 0;                         // 2 blocks, hi plane
constexpr int kTcALo = 2 * kBlockBytes;           // 2 blocks, lo plane
constexpr int kTcBHi = 4 * kBlockBytes;
constexpr int kTcBLo = 4 * kBlockBytes + kBBytes;
constexpr int kTcMisc = 4 * kBlockBytes + 2 * kBBytes;   // mbarrier, TMEM slot, max word
constexpr int kTcSmem = kTcMisc + 64;
constexpr int kTcStageLd = 9;                     // padded row (8 lines + 1) of the output staging
static_assert(1024 * kTcStageLd * 8 <= kTcMisc, "output staging must fit over the operands");

// Both DFT32 GEMMs of a 1024-point four-step transform of the 8 lines whose step-A
// operand (rows (line, n1), K = n2) is already in the A planes, scaled by `scale`.
// On return, warp w (line w) thread `lane` (k2) holds X[k2 + 32 k1] in x[k1]
// (unscaled).  `tmem` holds 128 columns; `phase` is the barrier's next parity
// (two phases are consumed).
// NBLK = 2: 8 lines (all warps hold a line); NBLK = 1: 4 lines (warps 0-3), the
// other warps only join the barriers.  bhi/blo: byte offsets of the DFT32 planes.
template <int SIGN, int NBLK = 2>
__device__ __forceinline__ void fft1024_gemms(char* sm, uint32_t tmem, uint64_t* bar, uint32_t phase, float scale,
                                              const float2* __restrict__ tw, int* err, float2 (&x)[32],
                                              int bhi = kTcBHi, int blo = kTcBLo) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int blk = warp >> 2, quad = warp & 3;
  const bool active = blk < NBLK;
  unsigned* maxw = reinterpret_cast<unsigned*>(sm + kTcMisc + 12);
  const uint32_t base = smem_u32(sm);
  // ---- step A: DFT32 over n2 for every row (line, n1)
  fence_proxy_async();
  fence_before_sync();
  __syncthreads();
  if (tid == 0) {
    fence_after_sync();
    issue_dft_gemm(tmem, base + kTcAHi, base + kTcALo, base + bhi, base + blo);
    if (NBLK == 2)
      issue_dft_gemm(tmem + 64, base + kTcAHi + kBlockBytes, base + kTcALo + kBlockBytes, base + bhi, base + blo);
    mma_commit(bar);
  }
  mbar_wait_bounded(bar, phase, err, 2);
  fence_after_sync();
  // row (line = warp, n1 = lane): Y[n1][k2] for k2 = 0..31 in columns 64*blk + 2k2 (+1)
  float y[64];
  const uint32_t lane_base = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(64 * blk);
  if (active) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_ld16(lane_base + 16 * c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) y[16 * c + i] = v[i];
    }
    tmem_wait_ld();
  } else {
#pragma unroll
    for (int i = 0; i < 64; ++i) y[i] = 0.f;
  }
  // twiddle W_1024^{SIGN n1 k2}
  float mx = 0.f;
#pragma unroll
  for (int k2 = 0; k2 < 32; ++k2) {
    float2 w = __ldg(tw + ((lane * k2) & 1023));
    if (SIGN > 0) w.y = -w.y;
    const float re = y[2 * k2] * w.x - y[2 * k2 + 1] * w.y;
    const float im = y[2 * k2] * w.y + y[2 * k2 + 1] * w.x;
    y[2 * k2] = re;
    y[2 * k2 + 1] = im;
    mx = fmaxf(mx, fmaxf(fabsf(re), fabsf(im)));
  }
  const float scale2 = pow2_scale(cta_max(mx, maxw));
  fence_before_sync();
  __syncthreads();   // every warp has read its accumulator before step C overwrites it
  // ---- step C operand: rows (line, k2), K = n1 (this thread's lane)
  char* a_hi = sm + kTcAHi;
  char* a_lo = sm + kTcALo;
  if (active) {
#pragma unroll
    for (int k2 = 0; k2 < 32; ++k2)
      put_c(a_hi, a_lo, warp * 32 + k2, lane, y[2 * k2] * scale2, y[2 * k2 + 1] * scale2);
  }
  fence_proxy_async();
  fence_before_sync();
  __syncthreads();
  if (tid == 0) {
    fence_after_sync();
    issue_dft_gemm(tmem, base + kTcAHi, base + kTcALo, base + bhi, base + blo);
    if (NBLK == 2)
      issue_dft_gemm(tmem + 64, base + kTcAHi + kBlockBytes, base + kTcALo + kBlockBytes, base + bhi, base + blo);
    mma_commit(bar);
  }
  mbar_wait_bounded(bar, phase ^ 1u, err, 3);
  fence_after_sync();
  // row (line = warp, k2 = lane): X[k2 + 32 k1] in columns 64*blk + 2k1 (+1)
  const float inv = 1.f / (scale * scale2);   // exact: both are powers of two
  if (active) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_ld16(lane_base + 16 * c, v);
#pragma unroll
      for (int i = 0; i < 8; ++i) x[8 * c + i] = make_float2(v[2 * i] * inv, v[2 * i + 1] * inv);
    }
    tmem_wait_ld();
  }
}

// Standalone 2D-FFT pass over 8 lines of a 1024 x 1024 field: AXIS 0 = rows
// (contiguous), AXIS 1 = columns.  Forward unscaled, inverse scaled 1/N per pass,
// as the FP32 passes (fft.js:58-59).
template <int AXIS, int SIGN>
__global__ void __launch_bounds__(kTcThreads) k_fft_tc(float2* data, const float2* __restrict__ tw, int* err) {
  constexpr int N = 1024;
  extern __shared__ __align__(1024) char sm[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kTcMisc);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kTcMisc + 8);
  unsigned* maxw = reinterpret_cast<unsigned*>(sm + kTcMisc + 12);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int l0 = blockIdx.x * kTcLines;
  if (warp == 0) {
    tmem_alloc(tslot, 128);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  build_dft32<SIGN>(sm + kTcBHi, sm + kTcBLo, tw);
  // load: thread (line g, n1 t) takes x[t + 32 n2] for n2 = 0..31 -- one whole operand row
  const int g = AXIS == 0 ? warp : (tid & 7), t = AXIS == 0 ? lane : (tid >> 3);
  float2 v[32];
  float mx = 0.f;
#pragma unroll
  for (int n2 = 0; n2 < 32; ++n2) {
    const int y = t + 32 * n2;
    v[n2] = AXIS == 0 ? data[(size_t)(l0 + g) * N + y] : data[(size_t)y * N + l0 + g];
    mx = fmaxf(mx, fmaxf(fabsf(v[n2].x), fabsf(v[n2].y)));
  }
  const float scale = pow2_scale(cta_max(mx, maxw));
#pragma unroll
  for (int n2 = 0; n2 < 32; ++n2) put_c(sm + kTcAHi, sm + kTcALo, g * 32 + t, n2, v[n2].x * scale, v[n2].y * scale);
  __syncthreads();   // the TMEM address written by warp 0 is visible to all
  const uint32_t tmem = *tslot;
  float2 x[32];
  fft1024_gemms<SIGN>(sm, tmem, bar, 0u, scale, tw, err, x);
  const float post = SIGN > 0 ? 1.f / N : 1.f;
  // stage through shared memory (over the operands, no longer read) for coalesced stores
  float2* st = reinterpret_cast<float2*>(sm);
  __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < 32; ++k1) {
    const int y = lane + 32 * k1;
    if (AXIS == 0) st[warp * (N + 1) + y] = make_float2(x[k1].x * post, x[k1].y * post);
    else st[y * kTcStageLd + warp] = make_float2(x[k1].x * post, x[k1].y * post);
  }
  __syncthreads();
#pragma unroll 4
  for (int i = tid; i < kTcLines * N; i += kTcThreads) {
    if (AXIS == 0) {
      const int gl = i / N, y = i - gl * N;
      data[(size_t)(l0 + gl) * N + y] = st[gl * (N + 1) + y];
    } else {
      const int y = i >> 3, gl = i & 7;
      data[(size_t)y * N + l0 + gl] = st[y * kTcStageLd + gl];
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, 128);
  }
}

// ---------------------------------------------------------------------------------------
// Fused physical-column stage at 1024^2 with both y-transforms on the tensor cores
// (the tcgen05 counterpart of k_phys_cols): a CTA owns 4 columns x0..x0+3.
//   lines 0-3 = PA columns, 4-7 = PB columns -> one 8-line inverse transform
//   warps 4-7 hand v(y) to warps 0-3 through shared memory
//   warps 0-3 form (u omega, v omega) -> one 4-line forward transform -> in-band Z rows
// MODE 0 = prime (velocity + speed only), 1 = stage, 2 = last stage (+ velocity, speed).
// Shared memory after the inverse transform (the operands are dead once its second
// GEMM has completed): v exchange over the block-1 hi plane, (u, v) staging over the
// block-1 lo plane and the inverse DFT32 planes, forward operands in block 0, Z
// staging over block 0.
constexpr int kTcCols = 4;
constexpr int kTcColsGrid = 1024 / kTcCols;
constexpr int kTcColsBHi = kTcSmem;                      // forward DFT32 planes, after the misc words
constexpr int kTcColsBLo = kTcSmem + kBBytes;
constexpr int kTcColsSmem = kTcSmem + 2 * kBBytes;
constexpr int kTcColsExch = kBlockBytes;                 // float [4][1024]
constexpr int kTcColsVel = 3 * kBlockBytes;              // float2 [1024][4], up to kTcMisc
static_assert(kTcColsVel + 1024 * kTcCols * 8 <= kTcMisc, "velocity staging overlaps the misc words");
static_assert(kTcColsBHi % 16 == 0, "descriptor base must be 16-byte aligned");

// (y, col) -> float2 slot of a [1024][4] staging tile; the XOR spreads a warp's
// fixed-column, consecutive-y writes over all banks
__device__ __forceinline__ int cols_stage_idx(int y, int col) { return 4 * y + (col ^ ((y >> 2) & 3)); }

template <int MODE>
__global__ void __launch_bounds__(kTcThreads, 2) k_phys_cols_tc(PhysArgs a, int* err) {
  constexpr int N = 1024;
  extern __shared__ __align__(1024) char sm[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kTcMisc);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kTcMisc + 8);
  unsigned* maxw = reinterpret_cast<unsigned*>(sm + kTcMisc + 12);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int x0 = blockIdx.x * kTcCols;
  if (warp == 0) {
    tmem_alloc(tslot, 128);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  build_dft32<+1>(sm + kTcBHi, sm + kTcBLo, a.tw);
  if (MODE != 0) build_dft32<-1>(sm + kTcColsBHi, sm + kTcColsBLo, a.tw);
  // load: thread (line g, n1 t) takes the pack at ky = t + 32 n2 -- one operand row
  const int g = tid & 7, t = tid >> 3;
  const float2* src = (g < kTcCols ? a.pa : a.pb) + x0 + (g & (kTcCols - 1));
  float2 v[32];
  float mx = 0.f;
#pragma unroll
  for (int n2 = 0; n2 < 32; ++n2) {
    v[n2] = __ldcs(src + (size_t)(t + 32 * n2) * N);
    mx = fmaxf(mx, fmaxf(fabsf(v[n2].x), fabsf(v[n2].y)));
  }
  const float scale = pow2_scale(cta_max(mx, maxw));
#pragma unroll
  for (int n2 = 0; n2 < 32; ++n2) put_c(sm + kTcAHi, sm + kTcALo, g * 32 + t, n2, v[n2].x * scale, v[n2].y * scale);
  __syncthreads();   // the TMEM address written by warp 0 is visible to all
  const uint32_t tmem = *tslot;
  float2 x[32];
  fft1024_gemms<+1, 2>(sm, tmem, bar, 0u, scale, a.tw, err, x);
  // warp w < 4: (omega, u) of column x0 + w at y = lane + 32 k1; warp 4 + w: (v, 0)
  float* sv = reinterpret_cast<float*>(sm + kTcColsExch);
  if (warp >= kTcCols) {
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) sv[(warp - kTcCols) * N + lane + 32 * k1] = x[k1].x;
  }
  __syncthreads();
  float speed = 0.f, mz = 0.f;
  float2* svel = reinterpret_cast<float2*>(sm + kTcColsVel);
  if (warp < kTcCols) {
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) {
      const int y = lane + 32 * k1;
      const float om = x[k1].x, u = x[k1].y, w = sv[warp * N + y];
      if (MODE != 1) {
        svel[cols_stage_idx(y, warp)] = make_float2(u, w);
        speed = fmaxf(speed, fabsf(u) + fabsf(w));
      }
      x[k1] = make_float2(u * om, w * om);
      mz = fmaxf(mz, fmaxf(fabsf(x[k1].x), fabsf(x[k1].y)));
    }
  }
  if (MODE != 0) {
    const float scale_z = pow2_scale(cta_max(mz, maxw));   // its barriers also publish svel
    if (MODE == 2) {
#pragma unroll 4
      for (int i = tid; i < N * kTcCols; i += kTcThreads) {
        const int y = i >> 2, c = i & 3;
        a.vel[(size_t)y * N + x0 + c] = svel[cols_stage_idx(y, c)];
      }
    }
    // forward operand: rows (line = warp, n1 = lane), K = n2 = k1 (block 0 only)
    if (warp < kTcCols) {
#pragma unroll
      for (int k1 = 0; k1 < 32; ++k1)
        put_c(sm + kTcAHi, sm + kTcALo, warp * 32 + lane, k1, x[k1].x * scale_z, x[k1].y * scale_z);
    }
    fft1024_gemms<-1, 1>(sm, tmem, bar, 0u, scale_z, a.tw, err, x, kTcColsBHi, kTcColsBLo);
    // warp w < 4: Z(ky = lane + 32 k1, x0 + w); stage for row-contiguous stores of the in-band rows
    float2* sz = reinterpret_cast<float2*>(sm);
    if (warp < kTcCols) {
#pragma unroll
      for (int k1 = 0; k1 < 32; ++k1) sz[cols_stage_idx(lane + 32 * k1, warp)] = x[k1];
    }
    __syncthreads();
#pragma unroll 4
    for (int i = tid; i < N * kTcCols; i += kTcThreads) {
      const int row = i >> 2, c = i & 3;
      if (fabsf(wn<N>(row)) < Tune<N>::KCUT) a.z[(size_t)row * N + x0 + c] = sz[cols_stage_idx(row, c)];
    }
  } else {
    __syncthreads();
#pragma unroll 4
    for (int i = tid; i < N * kTcCols; i += kTcThreads) {
      const int y = i >> 2, c = i & 3;
      a.vel[(size_t)y * N + x0 + c] = svel[cols_stage_idx(y, c)];
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, 128);
  }
  if (MODE != 1) cols_speed_finalize<kTcThreads>(a, speed);
}

}  // namespace tc
}  // namespace s2d
