// s2d_tc_cols.cuh -- the column stage at 1024^2 on the tensor cores, as independent
// warpgroup chains.
//
// A CTA owns 4 columns and runs two warpgroups (WG) that never wait for each other: WG g
// transforms columns x0 + 2g, x0 + 2g + 1 through its own operand buffer, its own 64 TMEM
// columns and its own MMA barrier, synchronising its 128 threads with a named barrier.
// The two WGs of a CTA and the two CTAs of an SM thus give four chains per SM that drift
// apart on the shared tensor core, so one chain's CUDA-core work (operand splits,
// twiddles, products) runs while another chain's GEMMs run.
//
// Per WG, both 1024-point y-transforms are four-step DFT-GEMMs (1024 = 32 x 32, split
// hi + lo FP16/BF16 operands, FP32 accumulation, see s2d_tc.cuh):
//   inverse: 4 lines (PA c0, PA c1, PB c0, PB c1) = one M = 128 block, K = 64 real
//   products u*omega + i v*omega of the 2 columns
//   forward: 2 lines = rows 0..63 of an M = 128 block (rows 64..127 are ignored)
// Only the forward DFT32 matrix and forward twiddles are held: the inverse transform is
// conj(F(conj x)), with the input conjugation folded into the operand scaling and the
// output conjugation into the final scaling (the middle twiddle needs none).
//
// Scaling: each step-A operand row carries its own power-of-two scale (known to the
// thread(s) that write the row, no reduction); the step-C rows mix values of every
// step-A row of a line and take the WG-wide bound 32 max|x| (|Y| <= sum |x|), read from
// per-warp maxima after the barrier that precedes the step-A GEMM anyway.
//
// Operand layout: K-major, no swizzle, core matrices of 8 rows x 16 bytes, K-adjacent
// core matrices LBO = 144 bytes apart (16 bytes past 128) and 8-row groups SBO = 1152
// bytes apart.  The extra 16 bytes put the K chunks of a row in different bank groups,
// and the step-C row orders below are chosen so that every transposition store of a
// warp (32 scalar stores, one per K position) hits 32 distinct banks.
#pragma once
#include "s2d_tc.cuh"

namespace s2d {
namespace tc {

constexpr int kC2Wg = 2;                          // warpgroups per CTA
constexpr int kC2Threads = 128 * kC2Wg;
constexpr int kC2Cols = 2 * kC2Wg;                // columns per CTA
constexpr int kC2Grid = 1024 / kC2Cols;
constexpr uint32_t kC2LBO = 144;
constexpr uint32_t kC2SBO = 8 * kC2LBO;           // 1152
constexpr int kC2Plane = 16 * kC2SBO;             // 128 rows x 64 halves: 18432 bytes
constexpr int kC2Op = 2 * kC2Plane;               // hi + lo
constexpr int kC2OffOp = 0;
constexpr int kC2OffB = kC2Wg * kC2Op;            // forward DFT32 hi | lo, then the twiddle matrix
constexpr int kC2OffTw = kC2OffB + 2 * kBBytes;
constexpr int kC2OffMisc = kC2OffTw + kTcTwBytes;
// misc words: setup barrier, TMEM base, per-WG MMA barriers, row-flag bitmask (32 words),
// per-warp maxima (8), per-row forward scales (2 WGs x 64)
constexpr int kC2MiscSetup = 0, kC2MiscTmem = 8, kC2MiscBar = 16, kC2MiscFlags = 32, kC2MiscMax = 160,
              kC2MiscRowScale = 192, kC2MiscBytes = 192 + 4 * 64 * kC2Wg;
constexpr int kC2Smem = kC2OffMisc + kC2MiscBytes;
static_assert(kC2OffB % 1024 == 0 && kC2OffTw % 16 == 0 && kC2OffMisc % 16 == 0, "alignment of the smem plan");
static_assert(15 * kC2SBO + 7 * kC2LBO + 128 <= kC2Plane, "core matrices stay inside their plane");
static_assert(2 * kC2Smem + 2048 <= 228 * 1024, "two CTAs per SM");

__device__ __forceinline__ uint32_t c2_off(int r, int k) {
  return (uint32_t)((r >> 3) * kC2SBO + (k >> 3) * kC2LBO + (r & 7) * 16 + (k & 7) * 2);
}

// one complex (re, im) at operand row r, complex column j, split into the hi / lo planes
template <class P>
__device__ __forceinline__ void c2_put1(char* op, int r, int j, float re, float im) {
  typename P::H2 h, l;
  split2<P>(re, im, h, l);
  const uint32_t o = c2_off(r, 2 * j);
  *reinterpret_cast<typename P::H2*>(op + o) = h;
  *reinterpret_cast<typename P::H2*>(op + kC2Plane + o) = l;
}
// four consecutive complex values (one 16-byte core-matrix row) at complex column 4 kc,
// as (re sr, im si) each
template <class P>
__device__ __forceinline__ void c2_put4(char* op, int r, int kc, const float2* v, float sr, float si) {
  typename P::H2 h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) split2<P>(v[i].x * sr, v[i].y * si, h[i], l[i]);
  const uint32_t o = c2_off(r, 8 * kc);
  *reinterpret_cast<uint4*>(op + o) = make_uint4(h2bits(h[0]), h2bits(h[1]), h2bits(h[2]), h2bits(h[3]));
  *reinterpret_cast<uint4*>(op + kC2Plane + o) = make_uint4(h2bits(l[0]), h2bits(l[1]), h2bits(l[2]), h2bits(l[3]));
}

// D[128 x 64] = A[128 x 64] . B over K = 64: hi.hi + hi.lo + lo.hi, 12 MMAs (K = 16 each)
template <class P>
__device__ __forceinline__ void c2_gemm(uint32_t tmem_d, uint32_t a, uint32_t b) {
  constexpr uint32_t idesc = idesc_f16(128, 64, P::kFmt);
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    const uint32_t ao = (uint32_t)kb * 2 * kC2LBO, bo = (uint32_t)kb * 2 * kLBO;
    const uint64_t ah = smem_desc(a + ao, kC2LBO, kC2SBO), al = smem_desc(a + kC2Plane + ao, kC2LBO, kC2SBO);
    const uint64_t bh = smem_desc(b + bo, kLBO, kSBO), bl = smem_desc(b + kBBytes + bo, kLBO, kSBO);
    mma_f16(tmem_d, ah, bh, idesc, kb > 0 ? 1u : 0u);
    mma_f16(tmem_d, ah, bl, idesc, 1u);
    mma_f16(tmem_d, al, bh, idesc, 1u);
  }
}

// named barrier of 128 threads (ids 1, 2 for the two WGs; 0 is __syncthreads), OR-reducing `pred`
template <int ID> __device__ __forceinline__ bool bar_or_128(bool pred) {
  uint32_t out;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, 128, p;\n selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(out)
      : "r"((uint32_t)pred), "n"(ID)
      : "memory");
  return out != 0;
}
__device__ __forceinline__ bool wg_bar_or(int wg, bool pred) {   // wg is warp-uniform
  return wg == 0 ? bar_or_128<1>(pred) : bar_or_128<2>(pred);
}

// 64 consecutive TMEM columns of this thread's lane
__device__ __forceinline__ void c2_tmem_read64(uint32_t addr, float (&y)[64]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    float v[16];
    tmem_ld16(addr + 16 * c, v);
#pragma unroll
    for (int i = 0; i < 16; ++i) y[16 * c + i] = v[i];
  }
  tmem_wait_ld();
}

// Step-A output row (fixed index n1 of one line) -> twiddled step-C operand column n1:
// T[k2] = D[k2] W_1024^{n1 k2} f for k2 = 0..31 into row row_of(k2).
template <class P, class RowOf>
__device__ __forceinline__ void c2_twiddle_scatter(const float (&y)[64], const char* sm, char* op, int n1, float f,
                                                   RowOf row_of) {
  const float4* trow = reinterpret_cast<const float4*>(sm + kC2OffTw + n1 * kTcTwLd * 8);
#pragma unroll
  for (int j = 0; j < 32; j += 2) {
    const float4 t4 = trow[j / 2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int k2 = j + e;
      const float wx = e ? t4.z : t4.x, wy = e ? t4.w : t4.y;
      const float re = (y[2 * k2] * wx - y[2 * k2 + 1] * wy) * f;
      const float im = (y[2 * k2] * wy + y[2 * k2 + 1] * wx) * f;
      c2_put1<P>(op, row_of(k2), n1, re, im);
    }
  }
}

// MMA issue by thread 0 of the WG after the WG barrier: fence the operand writes into the
// async proxy, synchronise, order after the barrier, issue, commit to the WG's barrier.
// Returns the agreed abort flag (some thread of the WG saw a wait give up).
template <class P>
__device__ __forceinline__ bool c2_issue(int wg, int wt, bool bad, uint32_t tmem_d, uint32_t a, uint32_t b,
                                         uint64_t* bar) {
  fence_proxy_async();
  fence_before_sync();
  const bool abort = wg_bar_or(wg, bad);
  if (!abort && wt == 0) {
    fence_after_sync();
    c2_gemm<P>(tmem_d, a, b);
    mma_commit(bar);
  }
  return abort;
}

template <int MODE, class P = PrecF16>
__global__ void __launch_bounds__(kC2Threads, 2) k_phys_cols_tc2(PhysArgs a, const char* __restrict__ tab, int* err) {
  constexpr int N = 1024;
  extern __shared__ __align__(1024) char sm[];
  char* misc = sm + kC2OffMisc;
  uint64_t* setup = reinterpret_cast<uint64_t*>(misc + kC2MiscSetup);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(misc + kC2MiscTmem);
  uint32_t* flags = reinterpret_cast<uint32_t*>(misc + kC2MiscFlags);
  float* wmax = reinterpret_cast<float*>(misc + kC2MiscMax);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wg = tid >> 7, wt = tid & 127;
  uint64_t* bar = reinterpret_cast<uint64_t*>(misc + kC2MiscBar) + wg;
  float* rowscale = reinterpret_cast<float*>(misc + kC2MiscRowScale) + 64 * wg;
  char* op = sm + kC2OffOp + wg * kC2Op;
  const uint32_t op_s = smem_u32(op), b_s = smem_u32(sm + kC2OffB);
  const int x0 = blockIdx.x * kC2Cols + 2 * wg;
  phys_latch(a);

  // ---- CTA set-up: TMEM (64 columns per WG), barriers, table copies, row-flag bitmask
  if (warp == 0) {
    tmem_alloc(tslot, 64 * kC2Wg);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(setup, 1);
    for (int g = 0; g < kC2Wg; ++g) mbar_init(reinterpret_cast<uint64_t*>(misc + kC2MiscBar) + g, 1);
    mbar_fence_init();
    mbar_arrive_expect_tx(setup, 2 * kBBytes + kTcTwBytes);
    bulk_g2s(sm + kC2OffB, tab + kTabFwd, 2 * kBBytes + kTcTwBytes, setup);   // DFT planes + twiddles
  }
  if (a.row_nz) {
#pragma unroll
    for (int i = 0; i < N / kC2Threads; ++i) {
      const int row = tid + kC2Threads * i;
      const unsigned bits = __ballot_sync(0xffffffffu, __ldg(a.row_nz + row) != 0);
      if (lane == 0) flags[row >> 5] = bits;
    }
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot + 64u * wg;
  const uint32_t trow_addr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);   // this thread's TMEM lane

  bool bad = false;      // a bounded wait of this thread gave up
  bool abort = false;    // agreed over the WG at each barrier
  uint32_t phase = 0;    // next phase of the WG's MMA barrier
  uint32_t issued = 2u;  // parity of the last GEMM issued by this WG (2 = none yet)
  float speed = 0.f;

  {
    // ---- inverse, step A operand: row wt = (n1, line), line 0/1 = PA col 0/1, 2/3 = PB col 0/1
    const int n1 = wt >> 2, line = wt & 3;
    const float2* src = (line < 2 ? a.pa : a.pb) + x0 + (line & 1);
    float2 v[32];
    float mx = 0.f;
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2) {
      const bool nz = a.row_nz ? ((flags[n2] >> n1) & 1u) : true;
      v[n2] = nz ? __ldcs(src + (size_t)(n1 + 32 * n2) * N) : make_float2(0.f, 0.f);
      mx = fmaxf(mx, fmaxf(fabsf(v[n2].x), fabsf(v[n2].y)));
    }
    const float sA = pow2_scale(mx);
#pragma unroll
    for (int kc = 0; kc < 8; ++kc) c2_put4<P>(op, wt, kc, &v[4 * kc], sA, -sA);   // conj: inverse via F
    mx = warp_max(mx);
    if (lane == 0) wmax[warp] = mx;
    // the table copies must have landed before the first GEMM reads them
    if (wt == 0) bad |= !mbar_wait_bounded(setup, 0u, err, 4);
    abort = c2_issue<P>(wg, wt, bad, tmem, op_s, b_s, bar);
    if (abort) goto done;
    issued = phase;

    // ---- step A done: twiddle into the step-C operand, row (k2, line) = 8 (k2/2) + 2 line + k2%2
    const float mall = fmaxf(fmaxf(wmax[4 * wg], wmax[4 * wg + 1]), fmaxf(wmax[4 * wg + 2], wmax[4 * wg + 3]));
    const float sC = pow2_scale(mall) * 0.03125f;
    bad |= !mbar_wait_bounded(setup, 0u, err, 4);                      // twiddles (already complete)
    bad |= !mbar_wait_bounded(bar, phase, err, 2);
    phase ^= 1u;
    fence_after_sync();
    float y[64];
    c2_tmem_read64(trow_addr, y);
    c2_twiddle_scatter<P>(y, sm, op, n1, sC / sA,
                          [&](int k2) { return 8 * (k2 >> 1) + 2 * line + (k2 & 1); });
    abort = c2_issue<P>(wg, wt, bad, tmem, op_s, b_s, bar);
    if (abort) goto done;
    issued = phase;

    // ---- step C done: thread row wt = (k2, line), x[k1] at y = k2 + 32 k1 (conj, unscaled)
    bad |= !mbar_wait_bounded(bar, phase, err, 3);
    phase ^= 1u;
    fence_after_sync();
    c2_tmem_read64(trow_addr, y);
    const int k2 = 2 * (wt >> 3) + (wt & 1), lc = (wt >> 1) & 3;
    const bool is_pa = lc < 2;
    const int col = lc & 1;
    const float inv = 1.f / sC;   // exact (power of two)
    // PA lane: (omega, u) at y; PB lane: (v, ~0).  The partner line (PA <-> PB of the same
    // column) is lane ^ 4.  The PA lane forms the products of k1 = 0..15, the PB lane of
    // k1 = 16..31 -- the two halves of the forward operand row (n1' = k2, col).
    float2 z[16];
    float mz = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float2 lo = make_float2(y[2 * k] * inv, -y[2 * k + 1] * inv);                 // k1 = k
      const float2 hi = make_float2(y[2 * (16 + k)] * inv, -y[2 * (16 + k) + 1] * inv);   // k1 = 16 + k
      const float2 send = is_pa ? hi : lo;
      const float rx = __shfl_xor_sync(0xffffffffu, send.x, 4);
      const float ry = __shfl_xor_sync(0xffffffffu, send.y, 4);
      // PA: omega, u = own lo, v = partner's lo.x;  PB: omega, u = partner's hi, v = own hi.x
      const float om = is_pa ? lo.x : rx, u = is_pa ? lo.y : ry, w = is_pa ? rx : hi.x;
      if constexpr (MODE != 1) {
        const int yy = k2 + 32 * (is_pa ? k : 16 + k);
        a.vel[(size_t)yy * N + x0 + col] = make_float2(u, w);
        speed = fmaxf(speed, fabsf(u) + fabsf(w));
      }
      z[k] = make_float2(u * om, w * om);
      mz = fmaxf(mz, fmaxf(fabsf(z[k].x), fabsf(z[k].y)));
    }
    if constexpr (MODE != 0) {
      // ---- forward, step A operand: row (n1' = k2, col) = 2 k2 + col; PA lane K chunks 0-3,
      // PB lane 4-7; the row's scale from the pair's maximum
      const float mrow = fmaxf(mz, __shfl_xor_sync(0xffffffffu, mz, 4));
      const float sF = pow2_scale(mrow);
      const int rf = 2 * k2 + col;
      if (is_pa) rowscale[rf] = sF;
#pragma unroll
      for (int q = 0; q < 4; ++q) c2_put4<P>(op, rf, (is_pa ? 0 : 4) + q, &z[4 * q], sF, sF);
      const float mw = warp_max(mz);
      if (lane == 0) wmax[warp] = mw;   // the WG's step-A maxima were read before the last barrier
      abort = c2_issue<P>(wg, wt, bad, tmem, op_s, b_s, bar);
      if (abort) goto done;
      issued = phase;
      const float mzall = fmaxf(fmaxf(wmax[4 * wg], wmax[4 * wg + 1]), fmaxf(wmax[4 * wg + 2], wmax[4 * wg + 3]));
      const float sCf = pow2_scale(mzall) * 0.03125f;
      if (wt < 64) {
        // ---- forward step A done (rows 0..63): row wt = (n1' = wt/2, col' = wt%2);
        // step-C row (k2'', col') = 8 (k2''/4) + 4 col' + k2''%4
        bad |= !mbar_wait_bounded(bar, phase, err, 2);
        fence_after_sync();
        c2_tmem_read64(trow_addr, y);
        const int n1f = wt >> 1, cf = wt & 1;
        c2_twiddle_scatter<P>(y, sm, op, n1f, sCf / rowscale[wt],
                              [&](int kk) { return 8 * (kk >> 2) + 4 * cf + (kk & 3); });
      }
      phase ^= 1u;
      abort = c2_issue<P>(wg, wt, bad, tmem, op_s, b_s, bar);
      if (abort) goto done;
      issued = phase;
      if (wt < 64) {
        // ---- forward step C done: row wt = (k2'' = 4 (wt/8) + wt%4, col'' = (wt/4)%2),
        // X[k2'' + 32 k1]; in-band rows of Z stored
        bad |= !mbar_wait_bounded(bar, phase, err, 3);
        fence_after_sync();
        c2_tmem_read64(trow_addr, y);
        const int kz = 4 * (wt >> 3) + (wt & 3), cz = (wt >> 2) & 1;
        const float invf = 1.f / sCf;
#pragma unroll
        for (int k1 = 0; k1 < 32; ++k1) {
          const int row = kz + 32 * k1;
          if (fabsf(wn<N>(row)) < Tune<N>::KCUT)
            a.z[(size_t)row * N + x0 + cz] = make_float2(y[2 * k1] * invf, y[2 * k1 + 1] * invf);
        }
      }
      phase ^= 1u;
    }
  }
done:
  // a WG that gave up may still have a GEMM or the table copies in flight: wait for them
  // (bounded) before the TMEM and shared memory they write are released
  if (__syncthreads_or(bad ? 1 : 0)) {
    if (tid == 0) mbar_wait_bounded(setup, 0u, nullptr, 0);
    if (wt == 0 && issued < 2u) mbar_wait_bounded(bar, issued, nullptr, 0);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(*tslot, 64 * kC2Wg);
  }
  if constexpr (MODE != 1) cols_speed_finalize<kC2Threads>(a, speed);
}

}  // namespace tc
}  // namespace s2d

namespace s2d {
namespace tc {

// ---------------------------------------------------------------------------------------
// The spectral-row stage at 1024^2 on the tensor cores (the tcgen05 counterpart of
// k_spec_rows), in the same warpgroup-chain form: a CTA runs two WGs, WG g owns the row
// pair p = 2 blockIdx.x + g (rows p and N - p; pair 0 is rows 0 and N/2).
//   forward x-transform of the two Z rows (rows 0..63 of an M = 128 block, line-major:
//     row = line * 32 + n1, so a warp's loads are consecutive in x)
//   Z_hat staged in natural order in the WG's operand buffer; all 128 threads then unpack
//     (partner row, Hermitian), form N_hat with the 2/3 mask, add forcing, apply the
//     integrating-factor RK3 stage update and form the next packs: thread (row line,
//     n1 = lane, n2 half) holds the cells kx = n1 + 32 n2 -- exactly its part of the
//     inverse transform's step-A operand rows, so no transposition is needed
//   inverse x-transform of the 4 pack lines (PA, PB of both rows; one M = 128 block),
//     written to PA / PB rows with lane-consecutive x
// The WG-wide power-of-two scale of the packs is read after the barrier that also
// decides whether both rows are all zero (then the inverse and its stores are skipped
// and the rows flagged, as the FP32 kernel does).
template <int MODE, bool PTR, class P = PrecF16>
__global__ void __launch_bounds__(kC2Threads, 2) k_spec_rows_tc2(SpecArgs a, const char* __restrict__ tab) {
  constexpr int N = 1024;
  constexpr float KCUT = Tune<N>::KCUT;
  extern __shared__ __align__(1024) char sm[];
  char* misc = sm + kC2OffMisc;
  uint64_t* setup = reinterpret_cast<uint64_t*>(misc + kC2MiscSetup);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(misc + kC2MiscTmem);
  float* wmax = reinterpret_cast<float*>(misc + kC2MiscMax);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wg = tid >> 7, wt = tid & 127, wq = warp & 3;
  uint64_t* bar = reinterpret_cast<uint64_t*>(misc + kC2MiscBar) + wg;
  int* s_nz = reinterpret_cast<int*>(misc + kC2MiscRowScale) + 8 * wg;   // per-warp "row holds a nonzero"
  char* op = sm + kC2OffOp + wg * kC2Op;
  float2* zs = reinterpret_cast<float2*>(op);                             // Z_hat staging [2][N]
  const uint32_t op_s = smem_u32(op), b_s = smem_u32(sm + kC2OffB);
  int* err = a.err;
  const int pair = blockIdx.x * kC2Wg + wg;
  const int row0 = pair == 0 ? 0 : pair, row1 = pair == 0 ? N / 2 : N - pair;
  auto row_of_line = [&](int l) { return l ? row1 : row0; };   // selects, not an indexed array

  if (warp == 0) {
    tmem_alloc(tslot, 64 * kC2Wg);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(setup, 1);
    for (int g = 0; g < kC2Wg; ++g) mbar_init(reinterpret_cast<uint64_t*>(misc + kC2MiscBar) + g, 1);
    mbar_fence_init();
    mbar_arrive_expect_tx(setup, 2 * kBBytes + kTcTwBytes);
    bulk_g2s(sm + kC2OffB, tab + kTabFwd, 2 * kBBytes + kTcTwBytes, setup);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot + 64u * wg;
  const uint32_t trow_addr = tmem + ((uint32_t)(32 * wq) << 16);

  bool bad = false, abort = false;
  uint32_t phase = 0, issued = 2u;
  // the first pair has the smallest |ky|: the WG is uniformly in or out of band work
  const bool any_band = MODE >= 0 && (float)pair < KCUT;
  // this thread's cells: row line `ln`, x = n1 + 32 n2 for n2 in [16 h, 16 h + 16)
  const int ln = wq & 1, n1 = lane, h = wq >> 1;
  const int row = row_of_line(ln);
  const float ky = wn<N>(row);
  const bool row_band = fabsf(ky) < KCUT;
  float2 nhat[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) nhat[j] = make_float2(0.f, 0.f);

  if (any_band) {
    // ---- forward x-transform of the two Z rows: step-A row wt = (line, n1), wt < 64
    float mx = 0.f, sA = 1.f;
    if (wt < 64) {
      const int zl = wt >> 5;
      const int zrow = row_of_line(zl);
      const bool zb = fabsf(wn<N>(zrow)) < KCUT;
      float2 v[32];
#pragma unroll
      for (int n2 = 0; n2 < 32; ++n2)
        v[n2] = zb ? __ldcs(a.z + (size_t)zrow * N + lane + 32 * n2) : make_float2(0.f, 0.f);
#pragma unroll
      for (int n2 = 0; n2 < 32; ++n2) mx = fmaxf(mx, fmaxf(fabsf(v[n2].x), fabsf(v[n2].y)));
      sA = pow2_scale(mx);
#pragma unroll
      for (int kc = 0; kc < 8; ++kc) c2_put4<P>(op, wt, kc, &v[4 * kc], sA, sA);
    }
    mx = warp_max(mx);
    if (lane == 0) wmax[warp] = mx;
    if (wt == 0) bad |= !mbar_wait_bounded(setup, 0u, err, 4);
    abort = c2_issue<P>(wg, wt, bad, tmem, op_s, b_s, bar);
    if (abort) goto done;
    issued = phase;
    {
      const float mall = fmaxf(wmax[4 * wg], wmax[4 * wg + 1]);
      const float sC = pow2_scale(mall) * 0.03125f;
      float y[64];
      if (wt < 64) {
        bad |= !mbar_wait_bounded(setup, 0u, err, 4);
        bad |= !mbar_wait_bounded(bar, phase, err, 2);
        fence_after_sync();
        c2_tmem_read64(trow_addr, y);
        const int zl = wt >> 5;
        c2_twiddle_scatter<P>(y, sm, op, lane, sC / sA, [&](int k2) { return 32 * zl + k2; });
      }
      phase ^= 1u;
      abort = c2_issue<P>(wg, wt, bad, tmem, op_s, b_s, bar);
      if (abort) goto done;
      issued = phase;
      if (wt < 64) {
        // step C done: row wt = (line, k2), X[k2 + 32 k1] into the natural-order staging
        bad |= !mbar_wait_bounded(bar, phase, err, 3);
        fence_after_sync();
        c2_tmem_read64(trow_addr, y);
        const int zl = wt >> 5;
        const float inv = 1.f / sC;
#pragma unroll
        for (int k1 = 0; k1 < 32; ++k1) zs[zl * N + lane + 32 * k1] = make_float2(y[2 * k1] * inv, y[2 * k1 + 1] * inv);
      }
      phase ^= 1u;
    }
    if (wg_bar_or(wg, bad)) goto done;   // staging visible to the WG
    {
      // ---- Hermitian unpack through the partner row, N_hat = i kx q1 + i ky q2, 2/3 mask
      const int pln = pair == 0 ? ln : ln ^ 1;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int c = n1 + 32 * (16 * h + j);
        const float kx = wn<N>(c);
        const float2 zk = zs[ln * N + c];
        const float2 zm = cconj(zs[pln * N + ((N - c) & (N - 1))]);
        const float2 q1 = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
        const float2 dd = csub(zk, zm);
        const float2 q2 = make_float2(0.5f * dd.y, -0.5f * dd.x);
        const bool band = row_band && fabsf(kx) < KCUT;
        nhat[j] = band ? make_float2(-(kx * q1.y) - ky * q2.y, kx * q1.x + ky * q2.x) : make_float2(0.f, 0.f);
      }
    }
    wg_bar_or(wg, false);                // staging reads done before the operand rewrites it
  }
  {
    // ---- RK3 stage update of this thread's 16 cells (solver.wgsl:97-122), next packs
    const DevParams& Pp = *a.params;
    float dt = 0.f;
    if constexpr (MODE >= 0) dt = __ldg(a.dt);
    const float2 fb2 = forcing_k2_bounds(Pp);
    constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
    const size_t rbase = (size_t)row * N;
    float2 pa[16], pb[16];
    float mp = 0.f;
    bool nzr = false;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int c = n1 + 32 * (16 * h + j);
      const float kx = wn<N>(c);
      const float k2 = kx * kx + ky * ky;
      const float2 wc = a.wcur[rbase + c];
      float2 w;
      if constexpr (MODE < 0) {
        w = wc;
      } else {
        const float2 w0 = MODE == 0 ? wc : a.w0[rbase + c];
        const bool band = row_band && fabsf(kx) < KCUT;
        float2 rhs = make_float2(-nhat[j].x, -nhat[j].y);
        if constexpr (PTR) {
          if (band) rhs = cadd(rhs, __ldg(a.fptr + rbase + c));
        }
        if (a.stochastic && band && k2 > 0.f && k2 >= fb2.x && k2 <= fb2.y)
          rhs = cadd(rhs, stochastic_term(Pp, N, row, c, kx, ky, k2, dt));
        const bool quiet = wc.x == 0.f && wc.y == 0.f && w0.x == 0.f && w0.y == 0.f && rhs.x == 0.f && rhs.y == 0.f;
        if (k2 == 0.f || quiet) w = make_float2(0.f, 0.f);
        else w = rk_update<MODE>(half_factor_m1(Pp, kx, k2, dt), w0, wc, rhs, dt);
        a.wout[rbase + c] = w;
      }
      nzr |= (w.x != 0.f || w.y != 0.f);
      const float inv = k2 > 0.f ? __frcp_rn(k2) : 0.f;
      const float fa = (1.f - ky * inv) * inv_n2;     // w + i u_hat = w (1 - ky/k2)
      const float fbk = kx * inv * inv_n2;            // v_hat = -i kx w / k2
      pa[j] = make_float2(w.x * fa, w.y * fa);
      pb[j] = make_float2(w.y * fbk, -w.x * fbk);
      mp = fmaxf(mp, fmaxf(fmaxf(fabsf(pa[j].x), fabsf(pa[j].y)), fmaxf(fabsf(pb[j].x), fabsf(pb[j].y))));
    }
    mp = warp_max(mp);
    const int wnz = __any_sync(0xffffffffu, nzr) ? 1 : 0;
    const int wbad = __any_sync(0xffffffffu, bad) ? 1 : 0;
    if (lane == 0) {
      wmax[warp] = mp;
      s_nz[wq] = wnz;
      s_nz[4 + wq] = wbad;
    }
    wg_bar_or(wg, false);
    // every thread reads the same words after the barrier: the decisions below are uniform
    const int nz0 = s_nz[0] | s_nz[2], nz1 = s_nz[1] | s_nz[3];
    const bool any_bad = (s_nz[4] | s_nz[5] | s_nz[6] | s_nz[7]) != 0;
    if (a.row_nz && wt == 0) {
      a.row_nz[row0] = nz0;
      a.row_nz[row1] = nz1;
    }
    if (any_bad) goto done;
    if (a.row_nz && !(nz0 | nz1)) goto done;   // both rows zero: no transforms, no stores (flagged)
    // ---- inverse x-transforms: step-A rows (line' = 2 ln + {PA, PB}) * 32 + n1, K chunks 4h..4h+3,
    // input conjugated (the inverse as conj(F(conj x)))
    const float mall = fmaxf(fmaxf(wmax[4 * wg], wmax[4 * wg + 1]), fmaxf(wmax[4 * wg + 2], wmax[4 * wg + 3]));
    const float sA = pow2_scale(mall);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      c2_put4<P>(op, (2 * ln) * 32 + n1, 4 * h + q, &pa[4 * q], sA, -sA);
      c2_put4<P>(op, (2 * ln + 1) * 32 + n1, 4 * h + q, &pb[4 * q], sA, -sA);
    }
    if (!any_band && wt == 0) bad |= !mbar_wait_bounded(setup, 0u, err, 4);   // first GEMM of this WG
    abort = c2_issue<P>(wg, wt, bad, tmem, op_s, b_s, bar);
    if (abort) goto done;
    issued = phase;
    const float sC = sA * 0.03125f;
    float y[64];
    bad |= !mbar_wait_bounded(setup, 0u, err, 4);
    bad |= !mbar_wait_bounded(bar, phase, err, 2);
    phase ^= 1u;
    fence_after_sync();
    c2_tmem_read64(trow_addr, y);
    {
      const int lp = wt >> 5;   // line' of this thread's step-A row (row wt = line' * 32 + n1)
      c2_twiddle_scatter<P>(y, sm, op, lane, 0.03125f, [&](int k2) { return 32 * lp + k2; });
    }
    abort = c2_issue<P>(wg, wt, bad, tmem, op_s, b_s, bar);
    if (abort) goto done;
    issued = phase;
    bad |= !mbar_wait_bounded(bar, phase, err, 3);
    phase ^= 1u;
    fence_after_sync();
    c2_tmem_read64(trow_addr, y);
    {
      // row wt = (line' = wt / 32, k2 = lane): conj(D) / sC at x = k2 + 32 k1
      const int lp = wt >> 5;
      float2* dst = ((lp & 1) ? a.pb : a.pa) + (size_t)row_of_line(lp >> 1) * N + lane;
      const float inv = 1.f / sC;
#pragma unroll
      for (int k1 = 0; k1 < 32; ++k1) dst[32 * k1] = make_float2(y[2 * k1] * inv, -y[2 * k1 + 1] * inv);
    }
  }
done:
  if (__syncthreads_or(bad ? 1 : 0)) {
    if (tid == 0) mbar_wait_bounded(setup, 0u, nullptr, 0);
    if (wt == 0 && issued < 2u) mbar_wait_bounded(bar, issued, nullptr, 0);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(*tslot, 64 * kC2Wg);
  }
}

}  // namespace tc
}  // namespace s2d
