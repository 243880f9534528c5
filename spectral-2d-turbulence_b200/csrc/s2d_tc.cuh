// s2d_tc.cuh -- tensor-core (tcgen05) DFT-GEMM line transforms for sm_100a.
//
// A 1024-point line is transformed in the four-step form N = 32 x 32:
//   x[n1 + 32 n2] --(DFT32 over n2, a GEMM)--> Y[n1][k2]
//   Y *= W_1024^{n1 k2}                        (FP32 twiddle, CUDA cores)
//   Y --(DFT32 over n1, a GEMM)--> X[k2 + 32 k1]
// Each DFT32 is a real GEMM D[M x 64] = A[M x 64] . B[64 x 64]: row r of A is
// (fixed index i, line l) with r = i * L + l for L lines, holding the 32 complex
// inputs as 64 interleaved (re, im) values along K; B is the real block form of
// the 32 x 32 DFT matrix.  The interleaved row order makes every operand store of
// a warp land in distinct shared-memory banks.
// Operands are split as hi + lo in FP16 (or BF16, the PrecBF16 instantiation) with
// x ~= hi + lo and the three products
// hi.hi + hi.lo + lo.hi accumulated in FP32 in tensor memory (TMEM).  A per-CTA
// power-of-two scale keeps the first GEMM's operand inside FP16 range; the
// second GEMM's operand is bounded by 32 x the first (|Y| <= sum |x|), so it
// takes that scale times 2^-5 without another reduction (scaling is exact).
//
// tcgen05 usage: one elected thread issues tcgen05.mma (cta_group::1,
// kind::f16, M = 128, N = 64, K = 16, A and B K-major in shared memory, no
// swizzle: 8 x 16-byte core matrices, LBO = 128 B between K-adjacent and
// SBO = 1024 B between M-adjacent core matrices), tcgen05.commit arrives on an
// mbarrier, and every warp reads its 32 TMEM lanes back with tcgen05.ld.
#pragma once
#include <cuda_bf16.h>
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
// fmt: operand format of A and B (0 = FP16, 1 = BF16), bits [7,10) and [10,13)
__host__ __device__ constexpr uint32_t idesc_f16(int m, int n, uint32_t fmt = 0) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// operand precision of the split: a pair type, its format code, pack and unpack
struct PrecF16 {
  using H2 = __half2;
  static constexpr uint32_t kFmt = 0;
  __device__ __forceinline__ static H2 pack(float a, float b) { return __floats2half2_rn(a, b); }
  __device__ __forceinline__ static float2 unpack(H2 v) { return __half22float2(v); }
};
struct PrecBF16 {
  using H2 = __nv_bfloat162;
  static constexpr uint32_t kFmt = 1;
  __device__ __forceinline__ static H2 pack(float a, float b) { return __floats2bfloat162_rn(a, b); }
  __device__ __forceinline__ static float2 unpack(H2 v) { return __bfloat1622float2(v); }
};

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

// split x into hi + lo with x ~= hi + lo
template <class P>
__device__ __forceinline__ void split2(float re, float im, typename P::H2& hi, typename P::H2& lo) {
  hi = P::pack(re, im);
  const float2 h = P::unpack(hi);
  lo = P::pack(re - h.x, im - h.y);
}
// store complex (re, im) at row r, complex column j (K = 2j, 2j+1) of the hi and lo planes
template <class P>
__device__ __forceinline__ void put_c(char* hi_plane, char* lo_plane, int r, int j, float re, float im) {
  typename P::H2 h, l;
  split2<P>(re, im, h, l);
  const uint32_t o = op_off(r, 2 * j);
  *reinterpret_cast<typename P::H2*>(hi_plane + o) = h;
  *reinterpret_cast<typename P::H2*>(lo_plane + o) = l;
}

// Real block form of the 32-point DFT with sign SIGN, stored transposed (row = output
// real index n, K = input real index): for output k2 and input n2, W = c + i s,
//   Bt[2k2][2n2] = c, Bt[2k2][2n2+1] = -s, Bt[2k2+1][2n2] = s, Bt[2k2+1][2n2+1] = c.
// W_32^{n2 k2} = W_1024^{32 n2 k2} from the FP64-generated twiddle table (forward sign).
template <int SIGN, class P>
__device__ __forceinline__ void build_dft32(char* hi_plane, char* lo_plane, const float2* __restrict__ tw1024) {
  for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
    const int k2 = e >> 5, n2 = e & 31;
    float2 w = __ldg(tw1024 + ((32 * n2 * k2) & 1023));
    if (SIGN > 0) w.y = -w.y;
    const float c = w.x, s = w.y;
    typename P::H2 h, l;
    // row 2k2: (c, -s) at K = 2n2, 2n2+1
    split2<P>(c, -s, h, l);
    uint32_t o = op_off(2 * k2, 2 * n2);
    *reinterpret_cast<typename P::H2*>(hi_plane + o) = h;
    *reinterpret_cast<typename P::H2*>(lo_plane + o) = l;
    // row 2k2+1: (s, c)
    split2<P>(s, c, h, l);
    o = op_off(2 * k2 + 1, 2 * n2);
    *reinterpret_cast<typename P::H2*>(hi_plane + o) = h;
    *reinterpret_cast<typename P::H2*>(lo_plane + o) = l;
  }
}

// D(block b) = A(block b) . B over K = 64: hi.hi + hi.lo + lo.hi, 3 x 4 MMAs of K = 16
template <class P>
__device__ __forceinline__ void issue_dft_gemm(uint32_t tmem_d, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi,
                                               uint32_t b_lo) {
  constexpr uint32_t idesc = idesc_f16(128, 64, P::kFmt);
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

// power-of-two scale that maps max |x| into [2^13, 2^14) (FP16 max is 65504), at most 2^126:
// a row of subnormal values (the far field of a localised vortex) would otherwise ask for
// a scale beyond FP32 range (inf, and inf * 0 = NaN); 2^126 and its inverse stay normal
__device__ __forceinline__ float pow2_scale(float maxabs) {
  if (!(maxabs > 0.f) || !isfinite(maxabs)) return 1.f;
  const int e = ilogbf(maxabs);                       // maxabs in [2^e, 2^(e+1))
  return ldexpf(1.f, min(13 - e, 126));
}

}  // namespace tc
}  // namespace s2d

namespace s2d {
namespace tc {

// ------------------------------------------------------------------ shared-memory plan
constexpr int kTcThreads = 256;                   // 8 warps
constexpr int kTcAHi = 0;                         // up to 2 M-blocks, hi plane
constexpr int kTcALo = 2 * kBlockBytes;           // up to 2 M-blocks, lo plane
constexpr int kTcBHi = 4 * kBlockBytes;           // inverse (+1) DFT32, hi / lo planes
constexpr int kTcBLo = 4 * kBlockBytes + kBBytes;
constexpr int kTcMisc = 4 * kBlockBytes + 2 * kBBytes;   // mbarriers, TMEM slot, per-warp max slots
constexpr int kTcFwdBHi = kTcMisc + 128;          // forward (-1) DFT32, hi / lo planes
constexpr int kTcFwdBLo = kTcFwdBHi + kBBytes;
constexpr int kTcTw = kTcFwdBLo + kBBytes;        // W_1024^{n1 k2}, rows n1 padded to 34 entries
constexpr int kTcTwLd = 34;                       // 272-byte rows: a warp's 4-8 rows start in distinct banks
constexpr int kTcTwBytes = 32 * kTcTwLd * 8;
constexpr int kTcSmem = kTcTw + kTcTwBytes;
static_assert(kTcFwdBHi % 16 == 0 && kTcTw % 16 == 0, "bulk-copy / descriptor bases must be 16-byte aligned");

// Global table (built once per solver by k_tc_tables, same byte layout as shared memory):
// [inverse DFT32 hi | lo][forward DFT32 hi | lo][twiddle matrix]
constexpr int kTabInv = 0;
constexpr int kTabFwd = 2 * kBBytes;
constexpr int kTabTw = 4 * kBBytes;
constexpr int kTabBytes = kTabTw + kTcTwBytes;

template <class P>
__global__ void k_tc_tables(char* tab, const float2* __restrict__ tw1024) {
  build_dft32<+1, P>(tab + kTabInv, tab + kTabInv + kBBytes, tw1024);
  build_dft32<-1, P>(tab + kTabFwd, tab + kTabFwd + kBBytes, tw1024);
  float2* t = reinterpret_cast<float2*>(tab + kTabTw);
  for (int e = threadIdx.x; e < 32 * kTcTwLd; e += blockDim.x) {
    const int n1 = e / kTcTwLd, k2 = e - n1 * kTcTwLd;
    t[e] = k2 < 32 ? tw1024[(n1 * k2) & 1023] : make_float2(0.f, 0.f);
  }
}

struct TcMisc {
  uint64_t* bar;     // GEMM completion
  uint32_t* tslot;
  float* red;        // [8] per-warp maxima
  uint64_t* setup;   // table bulk copies
};
__device__ __forceinline__ TcMisc tc_misc(char* sm) {
  return {reinterpret_cast<uint64_t*>(sm + kTcMisc), reinterpret_cast<uint32_t*>(sm + kTcMisc + 8),
          reinterpret_cast<float*>(sm + kTcMisc + 16), reinterpret_cast<uint64_t*>(sm + kTcMisc + 48)};
}

// One-time CTA setup: TMEM (128 columns), mbarriers, and TMA bulk copies of the DFT32
// planes of the signs used plus the twiddle matrix.  The barriers are visible to the
// other threads after the caller's next __syncthreads; tc_wait_tables before the
// first GEMM.
template <bool INV, bool FWD>
__device__ __forceinline__ void tc_setup(char* sm, const TcMisc& m, const char* __restrict__ tab) {
  if ((threadIdx.x >> 5) == 0) {
    tmem_alloc(m.tslot, 128);
    tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    mbar_init(m.bar, 1);
    mbar_init(m.setup, 1);
    mbar_fence_init();
    constexpr uint32_t bytes = (INV ? 2 * kBBytes : 0) + (FWD ? 2 * kBBytes : 0) + kTcTwBytes;
    mbar_arrive_expect_tx(m.setup, bytes);
    if (INV) bulk_g2s(sm + kTcBHi, tab + kTabInv, 2 * kBBytes, m.setup);
    if (FWD) bulk_g2s(sm + kTcFwdBHi, tab + kTabFwd, 2 * kBBytes + kTcTwBytes, m.setup);   // with the twiddles
    else bulk_g2s(sm + kTcTw, tab + kTabTw, kTcTwBytes, m.setup);
  }
}
__device__ __forceinline__ void tc_wait_tables(const TcMisc& m, int* err) { mbar_wait_bounded(m.setup, 0u, err, 4); }

// warp maximum into red[warp]; after a __syncthreads every thread reads the CTA max
__device__ __forceinline__ void warp_max_slot(float v, float* red) {
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
}
__device__ __forceinline__ float cta_max_slots(const float* red) {
  float m = red[0];
#pragma unroll
  for (int i = 1; i < kTcThreads / 32; ++i) m = fmaxf(m, red[i]);
  return m;
}

template <class H2> __device__ __forceinline__ uint32_t h2bits(H2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// four consecutive complex K values (one 16-byte core-matrix row) of operand row r,
// starting at complex index 4*kc, scaled by s, split into the hi and lo planes
template <class P>
__device__ __forceinline__ void put_c4(char* hi_plane, char* lo_plane, int r, int kc, float2 a, float2 b, float2 c,
                                       float2 d, float s) {
  typename P::H2 h0, h1, h2, h3, l0, l1, l2, l3;
  split2<P>(a.x * s, a.y * s, h0, l0);
  split2<P>(b.x * s, b.y * s, h1, l1);
  split2<P>(c.x * s, c.y * s, h2, l2);
  split2<P>(d.x * s, d.y * s, h3, l3);
  const uint32_t o = op_off(r, 8 * kc);
  *reinterpret_cast<uint4*>(hi_plane + o) = make_uint4(h2bits(h0), h2bits(h1), h2bits(h2), h2bits(h3));
  *reinterpret_cast<uint4*>(lo_plane + o) = make_uint4(h2bits(l0), h2bits(l1), h2bits(l2), h2bits(l3));
}

// Geometry of an L-line transform on 8 warps (L = 8: two M = 128 blocks, warp w reads
// block w / 4 whole; L = 4: one block, warps w and w + 4 read its columns 0-31 / 32-63).
// After either GEMM, thread (warp w, lane) owns TMEM row r = 128 blk + 32 (w & 3) + lane,
// i.e. fixed index r / L of line r % L, and NC = 16 * L / 4 complex columns from `col0`.
template <int L> struct TcGeom {
  static_assert(L == 4 || L == 8, "4 or 8 lines");
  static constexpr int NB = L / 4;                // M = 128 blocks
  static constexpr int NC = 16 * NB;              // complex columns a thread reads
  __device__ __forceinline__ static int row() {
    const int w = threadIdx.x >> 5;
    return (NB == 2 ? 128 * (w >> 2) : 0) + 32 * (w & 3) + (threadIdx.x & 31);
  }
  __device__ __forceinline__ static int line() { return row() % L; }
  __device__ __forceinline__ static int index() { return row() / L; }
  __device__ __forceinline__ static int col0() { return NB == 2 ? 0 : 16 * (int)(threadIdx.x >> 7); }
  __device__ __forceinline__ static uint32_t taddr(uint32_t tmem) {
    const int w = threadIdx.x >> 5;
    return tmem + ((uint32_t)(32 * (w & 3)) << 16) + (NB == 2 ? (uint32_t)(64 * (w >> 2)) : (uint32_t)(32 * (w >> 2)));
  }
};

template <int NC>
__device__ __forceinline__ void tmem_read(uint32_t addr, float (&y)[2 * NC]) {
#pragma unroll
  for (int c = 0; c < (2 * NC) / 16; ++c) {
    float v[16];
    tmem_ld16(addr + 16 * c, v);
#pragma unroll
    for (int i = 0; i < 16; ++i) y[16 * c + i] = v[i];
  }
  tmem_wait_ld();
}

template <class P>
__device__ __forceinline__ void issue_blocks(int nb, uint32_t tmem, uint32_t base, int bhi, int blo) {
  issue_dft_gemm<P>(tmem, base + kTcAHi, base + kTcALo, base + bhi, base + blo);
  if (nb == 2)
    issue_dft_gemm<P>(tmem + 64, base + kTcAHi + kBlockBytes, base + kTcALo + kBlockBytes, base + bhi, base + blo);
}

// Both DFT32 GEMMs of the 1024-point four-step transform of L lines whose step-A
// operand (row n1 * L + line, K = n2: x[n1 + 32 n2] * scale) the caller has written.
// On return the thread's TcGeom row is (k2 = index, line) and x[j] = X[k2 + 32 (col0 + j)],
// unscaled.  The barrier's next parity is `phase`; two phases are consumed.
template <int SIGN, int L, class P>
__device__ __forceinline__ void fft1024_gemms(char* sm, uint32_t tmem, uint64_t* bar, uint32_t phase, float scale,
                                              int* err, float2 (&x)[TcGeom<L>::NC]) {
  using G = TcGeom<L>;
  constexpr int NC = G::NC;
  const int bhi = SIGN > 0 ? kTcBHi : kTcFwdBHi, blo = SIGN > 0 ? kTcBLo : kTcFwdBLo;
  const uint32_t base = smem_u32(sm);
  // ---- step A: DFT32 over n2 for every row (n1, line)
  fence_proxy_async();
  fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_after_sync();
    issue_blocks<P>(G::NB, tmem, base, bhi, blo);
    mma_commit(bar);
  }
  mbar_wait_bounded(bar, phase, err, 2);
  fence_after_sync();
  float y[2 * NC];
  tmem_read<NC>(G::taddr(tmem), y);
  const int n1 = G::index(), line = G::line(), c0 = G::col0();
  // twiddle W_1024^{SIGN n1 k2}; step-C operand rows (k2, line), K = n1, at scale 2^-5
  // (the step-A GEMM has completed, so its operand planes are free; the accumulator is
  // only overwritten by the step-C GEMM, issued after every thread's TMEM read)
  char* a_hi = sm + kTcAHi;
  char* a_lo = sm + kTcALo;
  const float4* trow = reinterpret_cast<const float4*>(sm + kTcTw + n1 * kTcTwLd * 8) + c0 / 2;
#pragma unroll
  for (int j = 0; j < NC; j += 2) {
    const float4 t4 = trow[j / 2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int k2 = c0 + j + e;
      const float wx = e ? t4.z : t4.x, wy = SIGN > 0 ? -(e ? t4.w : t4.y) : (e ? t4.w : t4.y);
      const float re = (y[2 * (j + e)] * wx - y[2 * (j + e) + 1] * wy) * 0.03125f;
      const float im = (y[2 * (j + e)] * wy + y[2 * (j + e) + 1] * wx) * 0.03125f;
      put_c<P>(a_hi, a_lo, k2 * L + line, n1, re, im);
    }
  }
  fence_proxy_async();
  fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_after_sync();
    issue_blocks<P>(G::NB, tmem, base, bhi, blo);
    mma_commit(bar);
  }
  mbar_wait_bounded(bar, phase ^ 1u, err, 3);
  fence_after_sync();
  tmem_read<NC>(G::taddr(tmem), y);
  const float inv = 32.f / scale;   // exact: powers of two
#pragma unroll
  for (int j = 0; j < NC; ++j) x[j] = make_float2(y[2 * j] * inv, y[2 * j + 1] * inv);
}

__device__ __forceinline__ void tc_teardown(uint32_t tmem) {
  fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, 128);
  }
}

// ---------------------------------------------------------------------------------------
// Standalone 2D-FFT pass over 8 lines of a 1024 x 1024 field: AXIS 0 = rows
// (contiguous), AXIS 1 = columns.  Forward unscaled, inverse scaled 1/N per pass,
// as the FP32 passes (fft.js:58-59).
constexpr int kTcLines = 8;
constexpr int kTcRowLd = 1024 + 4;                // padded staging line (rows pass)
static_assert(kTcLines * kTcRowLd * 8 <= kTcMisc, "row staging must fit below the misc words");

template <int AXIS, int SIGN, class P = PrecF16>
__global__ void __launch_bounds__(kTcThreads) k_fft_tc(float2* data, const char* __restrict__ tab, int* err) {
  constexpr int N = 1024;
  extern __shared__ __align__(1024) char sm[];
  const TcMisc m = tc_misc(sm);
  const int tid = threadIdx.x;
  const int l0 = blockIdx.x * kTcLines;
  // load: thread (line g, n1 t) takes x[t + 32 n2], n2 = 0..31 -- one whole operand row
  const int g = tid & 7, t = tid >> 3;
  float2 v[32];
  float mx = 0.f;
#pragma unroll
  for (int n2 = 0; n2 < 32; ++n2) {
    const int y = t + 32 * n2;
    v[n2] = AXIS == 0 ? data[(size_t)(l0 + g) * N + y] : data[(size_t)y * N + l0 + g];
    mx = fmaxf(mx, fmaxf(fabsf(v[n2].x), fabsf(v[n2].y)));
  }
  tc_setup<(SIGN > 0), (SIGN < 0)>(sm, m, tab);
  warp_max_slot(mx, m.red);
  __syncthreads();
  const float scale = pow2_scale(cta_max_slots(m.red));
  const uint32_t tmem = *m.tslot;
#pragma unroll
  for (int kc = 0; kc < 8; ++kc)
    put_c4<P>(sm + kTcAHi, sm + kTcALo, t * kTcLines + g, kc, v[4 * kc], v[4 * kc + 1], v[4 * kc + 2],
              v[4 * kc + 3], scale);
  tc_wait_tables(m, err);
  float2 x[32];
  fft1024_gemms<SIGN, 8, P>(sm, tmem, m.bar, 0u, scale, err, x);
  const float post = SIGN > 0 ? 1.f / N : 1.f;
  // thread: line = lane & 7, k2; X[k2 + 32 k1] in x[k1].  Stage (over the dead operands)
  // for coalesced stores.
  // (both GEMMs have completed: operand and DFT planes are free)
  using G = TcGeom<8>;
  const int line = G::line(), k2 = G::index();
  float2* st = reinterpret_cast<float2*>(sm);
#pragma unroll
  for (int k1 = 0; k1 < 32; ++k1) {
    const int y = k2 + 32 * k1;
    const float2 o = make_float2(x[k1].x * post, x[k1].y * post);
    if (AXIS == 0) st[line * kTcRowLd + y] = o;
    else st[y * kTcLines + line] = o;
  }
  __syncthreads();
#pragma unroll 4
  for (int i = tid; i < kTcLines * N; i += kTcThreads) {
    if (AXIS == 0) {
      const int gl = i >> 10, y = i & (N - 1);
      data[(size_t)(l0 + gl) * N + y] = st[gl * kTcRowLd + y];
    } else {
      data[(size_t)(i >> 3) * N + l0 + (i & 7)] = st[i];
    }
  }
  tc_teardown(tmem);
}

}  // namespace tc
}  // namespace s2d
