// s2d_kernels.cuh -- sm_100a kernels of the integrating-factor RK3 step.
//
// Fused step (one RK stage = two kernels, both whole-line FFTs in shared memory):
//
//   k_phys_cols  "physical columns": for a tile of GA columns x, read the
//                x-transformed packs PA(ky,x) = FFT_x^-1(w + i u_hat),
//                PB(ky,x) = FFT_x^-1(v_hat), y-IFFT both to (omega, u, v)(y,x),
//                form u*omega + i v*omega, y-FFT it and store the dealiased rows
//                Z(ky,x) (|ky| < N/3 only).  At the last stage it also writes the
//                velocity (u,v) for the dye and reduces max|u|+|v| for the CFL dt.
//   k_spec_rows  "spectral row pairs": for the rows ky and -ky, x-FFT Z, unpack the
//                two real spectra through the partner row (Hermitian unpack),
//                form N_hat = i kx q1 + i ky q2 with the 2/3 mask, add pointer and
//                stochastic forcing, apply the integrating-factor RK3 stage update,
//                then pack the NEXT stage's (w + i u_hat, v_hat), scale 1/N^2 and
//                x-IFFT them into PA, PB.
//
// Per stage this moves ~45 N^2 bytes in k_spec_rows and ~21 N^2 in k_phys_cols
// instead of the reference's 7 full passes.  The standalone kernels at the end
// (velocity_pack, nl_pack, assemble, rk3, fft rows/cols) reproduce the
// reference's unfused stages one for one, for the per-stage test hooks.
#pragma once
#include "s2d_async.cuh"
#include "s2d_device.cuh"

namespace s2d {

// Launch shape of the stage kernels for N x N: V values per thread (T = N/V threads per
// line; the line FFT runs radix-V passes), GA columns per column-kernel CTA, PPB row pairs
// per row-kernel CTA, the resident CTAs the register budget must allow (AMB_/BMB_;
// 0 = as many as 128 registers a thread give), whether the row kernel stages the
// rows its RK update reads by bulk copy (PF_), and whether it runs the two inverse
// x-transforms of the next packs as one two-line transform (PAIR_: half the
// barrier-separated passes, twice the registers).  Tune<N> is the default shape; the
// autotuner picks among the variants each size registers (s2d_ops.cuh).
template <int N_, int V_ = 16, int AMB_ = 0, int BMB_ = 0, bool PF_ = false, bool PAIR_ = false> struct Tune {
  static constexpr int N = N_;
  static constexpr int V = V_;
  static constexpr int T = N / V;
  using PL = LinePlan<N, V>;
  // physical-column kernel: GA columns per CTA, lanes run over columns first
  static constexpr int GA = N >= 4096 ? 2 : ((256 / T) > 4 ? ((256 / T) < N ? (256 / T) : N) : 4);
  static constexpr int A_THREADS = GA * T;
  static constexpr int A_LDS = PL::stride(GA >= 16 ? 1 : 16 / GA);
  static constexpr int A_GRID = N / GA;
  // spectral-row kernel: PPB row pairs (2*PPB rows) per CTA, lanes run along a row
  static constexpr int PPB = T >= 64 ? 1 : ((64 / T) < N / 2 ? (64 / T) : N / 2);
  static constexpr int B_ROWS = 2 * PPB;
  static constexpr int B_THREADS = B_ROWS * T;
  static constexpr int B_LDS = PL::stride(T >= 16 ? 0 : T);
  static constexpr int B_GRID = (N / 2) / PPB;
  static constexpr float KCUT = (float)(N / 3.0);
  // resident CTAs the register budget must allow
  static constexpr int A_MINB = AMB_ ? AMB_ : (65536 / (A_THREADS * 128) > 0 ? 65536 / (A_THREADS * 128) : 1);
  static constexpr int B_MINB = BMB_ ? BMB_ : (65536 / (B_THREADS * 128) > 0 ? 65536 / (B_THREADS * 128) : 1);
  static constexpr size_t A_SMEM = sizeof(float2) * 2 * GA * A_LDS;
  static constexpr size_t B_SMEM = sizeof(float2) * 2 * B_ROWS * B_LDS;
  // PF_: the spectral-row kernel stages the rows its RK update reads (wcur, w0 from
  // stage 1 on, the pointer force when splats are active) by bulk copy into shared
  // memory after the exchange lines; they land while the Z loads and the x-FFT run.  The
  // staging is sized per kernel instance (spec_smem): 16 KB a row pair per array at
  // 1024^2, so the stage kernels without pointer forcing keep 3 CTAs per SM.
  static constexpr bool PREFETCH = PF_;
  static constexpr bool PAIR_IFFT = PAIR_;
  static constexpr size_t B_BAR_OFF = B_SMEM;
  static constexpr size_t B_STAGE_OFF = B_SMEM + 16;
  static constexpr size_t B_SMEM_TOTAL = B_STAGE_OFF;   // without staging
  static constexpr size_t COLS_SMEM = sizeof(float2) * GA * A_LDS;
  static constexpr size_t ROWS_SMEM = sizeof(float2) * B_ROWS * B_LDS;
};

struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// ---------------------------------------------------------------------------------------
// arguments of the fused kernels
struct PhysArgs {
  const float2* pa;     // x-transformed packs, [ky][x]
  const float2* pb;
  float2* z;            // product spectrum after the y-FFT, [ky][x], in-band rows
  float2* vel;          // physical (u, v), [y][x]
  float* partials;      // per-CTA max |u|+|v|
  unsigned* ticket;     // last-CTA-done counter
  float* dt_out;        // dt slot written by the last CTA: [dt, speed]
  const DevParams* params;
  const float2* tw;
  int reduce;           // finalize the CFL dt into dt_out
  DevParams* latch;     // non-null: latch step_index from *counter (and advance it) first
  uint32_t* counter;
  const int* row_nz;    // non-null: row ky of PA/PB is all zero (and need not be read) where 0
};

// the per-substep stepIndex latch (S2D_STEP_RELATCH): params.step_index = counter++,
// the step index a configure() before this substep would latch (solver.js:316); done by
// one thread of the first stage's column kernel, since nothing in that kernel reads
// step_index and its first reader (the row kernel's stochastic forcing) is the next launch
__device__ __forceinline__ void phys_latch(const PhysArgs& a) {
  if (a.latch && blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t k = *a.counter;
    a.latch->step_index = k;
    *a.counter = k + 1u;
  }
}

struct SpecArgs {
  const float2* z;      // product spectrum (ky, x), in-band rows
  const float2* w0;     // state at the start of the step
  const float2* wcur;   // state entering this stage (prime: the state to pack)
  float2* wout;         // state leaving this stage
  const float2* fptr;   // pointer-force spectrum, or nullptr
  float2* pa;           // next-stage packs, x-transformed, [ky][x]
  float2* pb;
  const float* dt;      // current dt slot
  const DevParams* params;
  const float2* tw;
  int stochastic;       // force_amp > 0
  int* err;             // device error word (bounded waits that gave up)
  int* row_nz;          // non-null: per row, 1 if the written PA/PB row holds a nonzero value;
                        // a CTA whose rows are all zero then skips its transforms and stores
};

// rows held by the 2*PPB row slots of tile `tile`: pair p = rows (p, N-p); pair 0 = rows (0, N/2)
template <int N, class TU = Tune<N>> __device__ __forceinline__ int spec_row_of(int tile, int slot) {
  const int pair = tile * TU::PPB + (slot >> 1);
  const int which = slot & 1;
  return pair == 0 ? (which ? N / 2 : 0) : (which ? N - pair : pair);
}

// number of staged row arrays for a stage: wcur, w0 (stages 1-2), pointer force
template <int MODE, bool PTR> __host__ __device__ constexpr int spec_stage_arrays() {
  return (MODE >= 1 ? 2 : 1) + (PTR ? 1 : 0);
}
// dynamic shared memory of one spectral-row kernel instance: exchange lines, tile
// barrier, then (PF_) the staged rows
template <class TU, int MODE, bool PTR> __host__ __device__ constexpr size_t spec_smem() {
  return TU::B_STAGE_OFF +
         (TU::PREFETCH ? sizeof(float2) * spec_stage_arrays<MODE, PTR>() * TU::B_ROWS * TU::N : 0);
}

// ---------------------------------------------------------------------------------------
// physical columns: MODE 0 = prime (velocity + speed only), 1 = stage, 2 = last stage
// (stage + velocity + speed)
// one tile of GA columns; returns this thread's max |u|+|v| (MODE != 1)
template <int N, int MODE, class TU = Tune<N>>
__device__ __forceinline__ float phys_cols_tile(const PhysArgs& a, int tile, float2* smem) {
  constexpr int V = TU::V, T = TU::T, GA = TU::GA, LDS = TU::A_LDS;
  const int tid = threadIdx.x;
  const int g = tid % GA, t = tid / GA;
  const int x = tile * GA + g;
  float2* const bufs[2] = {smem + g * LDS, smem + (GA + g) * LDS};

  float2 v[2][V];
  if (a.row_nz) {
    // rows the row kernel left unwritten (all zero) are not read
    int nz[V];
#pragma unroll
    for (int m = 0; m < V; ++m) nz[m] = __ldg(a.row_nz + t + T * m);
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const size_t o = (size_t)(t + T * m) * N + x;
      v[0][m] = nz[m] ? __ldcs(a.pa + o) : make_float2(0.f, 0.f);
      v[1][m] = nz[m] ? __ldcs(a.pb + o) : make_float2(0.f, 0.f);
    }
  } else {
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const size_t o = (size_t)(t + T * m) * N + x;
      v[0][m] = __ldcs(a.pa + o);
      v[1][m] = __ldcs(a.pb + o);
    }
  }
  fft_lines<N, V, +1, 2>(v, bufs, t, a.tw, CtaSync{});
  // v[0][m] = (omega, u), v[1][m].x = v at physical row y = t + T*m

  float speed = 0.f;
  if constexpr (MODE != 1) {
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const float u = v[0][m].y, w = v[1][m].x;
      a.vel[(size_t)(t + T * m) * N + x] = make_float2(u, w);
      speed = fmaxf(speed, fabsf(u) + fabsf(w));
    }
  }
  if constexpr (MODE != 0) {
    float2 z[1][V];
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const float om = v[0][m].x;
      z[0][m] = make_float2(v[0][m].y * om, v[1][m].x * om);
    }
    float2* const zb[1] = {bufs[0]};
    fft_lines<N, V, -1, 1>(z, zb, t, a.tw, CtaSync{});
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const int row = t + T * m;
      if (fabsf(wn<N>(row)) < TU::KCUT) a.z[(size_t)row * N + x] = z[0][m];
    }
  }
  return speed;
}

// CTA max of |u|+|v| into partials[blockIdx.x]; with a.reduce the last CTA to finish
// reduces the partials and writes [dt, speed] into a.dt_out (last-CTA-done ticket).
// Every thread of a CTA of NTHREADS calls it.
template <int NTHREADS>
__device__ __forceinline__ void cols_speed_finalize(const PhysArgs& a, float speed) {
  __shared__ float red[32];
  __shared__ int last;
  const int tid = threadIdx.x;
  speed = warp_max(speed);
  const int lane = tid & 31, warp = tid >> 5;
  if (lane == 0) red[warp] = speed;
  __syncthreads();
  if (warp == 0) {
    float s = lane < (NTHREADS + 31) / 32 ? red[lane] : 0.f;
    s = warp_max(s);
    if (lane == 0) {
      a.partials[blockIdx.x] = s;
      int is_last = 0;
      if (a.reduce) {
        __threadfence();
        const unsigned k = atomicAdd(a.ticket, 1u);
        is_last = (k == gridDim.x - 1);
      }
      last = is_last;
    }
  }
  __syncthreads();
  if (last) {
    __threadfence();   // acquire side of the ticket: the other CTAs' partials are read after it
    float s = 0.f;
    for (int i = tid; i < (int)gridDim.x; i += blockDim.x) s = fmaxf(s, __ldcg(a.partials + i));
    s = warp_max(s);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
      float m = 0.f;
      for (int i = 0; i < (NTHREADS + 31) / 32; ++i) m = fmaxf(m, red[i]);
      a.dt_out[0] = cfl_dt(*a.params, m);
      a.dt_out[1] = m;
      *a.ticket = 0u;
    }
  }
}

template <int N, int MODE, class TU = Tune<N>>
__global__ void __launch_bounds__(TU::A_THREADS, TU::A_MINB) k_phys_cols(PhysArgs a) {
  extern __shared__ float2 smem[];
  phys_latch(a);
  const float speed = phys_cols_tile<N, MODE, TU>(a, blockIdx.x, smem);
  if constexpr (MODE != 1) cols_speed_finalize<TU::A_THREADS>(a, speed);
}

// ---------------------------------------------------------------------------------------
// spectral row pairs: MODE -1 = prime (pack wcur only), 0/1/2 = RK stage
// `bar` is an initialised mbarrier in shared memory whose next phase is `parity`
// (one phase per call); it orders the TMA bulk copies of this tile's rows.
template <int N, int MODE, bool PTR, class TU = Tune<N>>
__device__ __forceinline__ void spec_rows_tile(const SpecArgs& a, int tile, float2* smem, uint64_t* bar,
                                               uint32_t parity) {
  constexpr int V = TU::V, T = TU::T, LDS = TU::B_LDS;
  constexpr float KCUT = TU::KCUT;
  constexpr int NARR = spec_stage_arrays<MODE, PTR>();
  const int tid = threadIdx.x;
  const int t = tid % T, slot = tid / T;
  const int pair = tile * TU::PPB + (slot >> 1);
  const int row = spec_row_of<N, TU>(tile, slot);
  const int pslot = pair == 0 ? slot : (slot ^ 1);
  float2* const stage = reinterpret_cast<float2*>(reinterpret_cast<char*>(smem) + TU::B_STAGE_OFF);
  if constexpr (TU::PREFETCH) {
    // one thread stages the rows this tile's RK update reads; they land while the
    // x-FFT of Z runs
    if (tid == 0) {
      mbar_arrive_expect_tx(bar, (uint32_t)(NARR * TU::B_ROWS * N * sizeof(float2)));
      for (int s = 0; s < TU::B_ROWS; ++s) {
        const size_t ro = (size_t)spec_row_of<N, TU>(tile, s) * N;
        int k = 0;
        bulk_g2s(stage + (size_t)(k++ * TU::B_ROWS + s) * N, a.wcur + ro, N * sizeof(float2), bar);
        if constexpr (MODE >= 1) bulk_g2s(stage + (size_t)(k++ * TU::B_ROWS + s) * N, a.w0 + ro, N * sizeof(float2), bar);
        if constexpr (PTR) bulk_g2s(stage + (size_t)(k++ * TU::B_ROWS + s) * N, a.fptr + ro, N * sizeof(float2), bar);
      }
    }
  }
  const float2* const s_wcur = stage + (size_t)slot * N;
  const float2* const s_w0 = stage + (size_t)(TU::B_ROWS + slot) * N;
  const float2* const s_fptr = stage + (size_t)((MODE >= 1 ? 2 : 1) * TU::B_ROWS + slot) * N;
  float2* const own0 = smem + (2 * slot) * LDS;
  float2* const own1 = smem + (2 * slot + 1) * LDS;
  const float ky = wn<N>(row);
  const bool row_band = fabsf(ky) < KCUT;
  const size_t rbase = (size_t)row * N;

  // own0: the exchange line of this row's transforms; own1: this row's N_hat, then
  // its updated state, in natural (padded) order -- each thread touches only the
  // slots of its own elements there, so own1 needs no barrier.
  using PL = LinePlan<N, V>;
  bool any_band = false;
  if constexpr (MODE >= 0) {
    // the first pair of this CTA has the smallest |ky|: the CTA is uniformly in/out of band work
    any_band = (float)(tile * TU::PPB) < KCUT;
    if (any_band) {
      float2 zz[1][V];
#pragma unroll
      for (int m = 0; m < V; ++m) zz[0][m] = row_band ? __ldcs(a.z + rbase + t + T * m) : make_float2(0.f, 0.f);
      float2* const zb[1] = {own0};
      fft_lines<N, V, -1, 1>(zz, zb, t, a.tw, CtaSync{});
#pragma unroll
      for (int m = 0; m < V; ++m) own0[PL::pad(t + T * m)] = zz[0][m];
      __syncthreads();
      const float2* pbuf = smem + (2 * pslot) * LDS;
#pragma unroll
      for (int m = 0; m < V; ++m) {
        const int c = t + T * m;
        const float kx = wn<N>(c);
        const float2 zk = zz[0][m];
        const float2 zm = cconj(pbuf[PL::pad((N - c) & (N - 1))]);
        // q1 = (Z_k + conj Z_-k)/2, q2 = -i (Z_k - conj Z_-k)/2 (solver.wgsl:68-72)
        const float2 q1 = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
        const float2 dd = csub(zk, zm);
        const float2 q2 = make_float2(0.5f * dd.y, -0.5f * dd.x);
        const bool band = row_band && fabsf(kx) < KCUT;
        // N_hat = kx * (i q1) + ky * (i q2)
        own1[PL::pad(c)] =
            band ? make_float2(-(kx * q1.y) - ky * q2.y, kx * q1.x + ky * q2.x) : make_float2(0.f, 0.f);
      }
      __syncthreads();   // partner reads of own0 done before the transforms below reuse it
    }
  }

  if constexpr (TU::PREFETCH) mbar_wait_bounded(bar, parity, a.err, 1);

  // per-row "holds a nonzero value" flags of this tile (only when the caller tracks them)
  __shared__ int s_nz[32];
  if (a.row_nz) {
    if (t == 0) s_nz[slot] = 0;
    __syncthreads();
  }
  bool row_nonzero = false;
  // RK3 stage update, one cell per iteration (unrolled by two only: the forcing and
  // integrating-factor code appears twice in the kernel, not V times; by two measured 3 %
  // faster than rolled at 1024^2 with no spills); the state
  // (and pointer-force) values of the next cell are loaded one iteration ahead so
  // their latency overlaps this cell's arithmetic
  {
    const DevParams& P = *a.params;
    float dt = 0.f;
    if constexpr (MODE >= 0) dt = __ldg(a.dt);
    const float2 fb = forcing_k2_bounds(P);
    const float2 zero2 = make_float2(0.f, 0.f);
    auto ld_wc = [&](int c) { return TU::PREFETCH ? s_wcur[c] : a.wcur[rbase + c]; };
    auto ld_w0 = [&](int c) { return TU::PREFETCH ? s_w0[c] : a.w0[rbase + c]; };
    auto ld_fp = [&](int c) { return TU::PREFETCH ? s_fptr[c] : __ldg(a.fptr + rbase + c); };
    float2 wc_next = ld_wc(t), w0_next = zero2, fp_next = zero2;
    if constexpr (MODE >= 1) w0_next = ld_w0(t);
    if constexpr (PTR && MODE >= 0) fp_next = ld_fp(t);
#pragma unroll 2
    for (int m = 0; m < V; ++m) {
      const int c = t + T * m;
      const size_t o = rbase + c;
      const float2 wc = wc_next;
      const float2 w0v = w0_next, fpv = fp_next;
      if (m + 1 < V) {
        wc_next = ld_wc(c + T);
        if constexpr (MODE >= 1) w0_next = ld_w0(c + T);
        if constexpr (PTR && MODE >= 0) fp_next = ld_fp(c + T);
      }
      float2 w;
      if constexpr (MODE < 0) {
        w = wc;
      } else {
        const float kx = wn<N>(c);
        const float k2 = kx * kx + ky * ky;
        const float2 w0 = MODE == 0 ? wc : w0v;
        const bool band = row_band && fabsf(kx) < KCUT;
        const float2 nhat = any_band ? own1[PL::pad(c)] : zero2;
        float2 rhs = make_float2(-nhat.x, -nhat.y);
        if constexpr (PTR) {
          if (band) rhs = cadd(rhs, fpv);
        }
        if (a.stochastic && band && k2 > 0.f && k2 >= fb.x && k2 <= fb.y)
          rhs = cadd(rhs, stochastic_term(P, N, row, c, kx, ky, k2, dt));
        // a cell whose state and right-hand side are all zero stays zero (every stage form
        // is linear in w0, wcur, rhs): the modes outside the dealias band of a dealiased
        // state skip the integrating factor
        const bool quiet = wc.x == 0.f && wc.y == 0.f && w0.x == 0.f && w0.y == 0.f && rhs.x == 0.f && rhs.y == 0.f;
        if (k2 == 0.f || quiet) w = zero2;
        else w = rk_update<MODE>(half_factor_m1(P, kx, k2, dt), w0, wc, rhs, dt);
        a.wout[o] = w;
      }
      own1[PL::pad(c)] = w;
      row_nonzero |= (w.x != 0.f || w.y != 0.f);
    }
  }
  if (a.row_nz) {
    if (row_nonzero) s_nz[slot] = 1;
    // all rows of the tile zero: their packs are zero -- flag them and skip the transforms
    // and stores (the column kernels read no flagged row)
    const int any = __syncthreads_or(row_nonzero ? 1 : 0);
    if (t == 0) a.row_nz[row] = s_nz[slot];
    if (!any) return;
  }

  // next-stage packs, scaled by the 1/N^2 of the inverse 2D transform, x-IFFT each;
  // the two transforms share one code path
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
  if constexpr (TU::PAIR_IFFT) {
    // both packs formed first, then one two-line transform through own0 and own1 (the
    // same arithmetic per line as the one-line transforms below)
    float2 x[2][V];
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const int c = t + T * m;
      const float kx = wn<N>(c);
      const float k2 = kx * kx + ky * ky;
      const float inv = k2 > 0.f ? __frcp_rn(k2) : 0.f;
      const float2 w = own1[PL::pad(c)];
      const float fa = (1.f - ky * inv) * inv_n2;       // w + i u_hat = w (1 - ky/k2)
      const float fb = kx * inv * inv_n2;                // v_hat = -i kx w / k2
      x[0][m] = make_float2(w.x * fa, w.y * fa);
      x[1][m] = make_float2(w.y * fb, -w.x * fb);
    }
    __syncthreads();   // every thread's own1 reads done before the transform writes own1
    float2* const xb[2] = {own0, own1};
    fft_lines<N, V, +1, 2>(x, xb, t, a.tw, CtaSync{});
#pragma unroll
    for (int m = 0; m < V; ++m) {
      a.pa[rbase + t + T * m] = x[0][m];
      a.pb[rbase + t + T * m] = x[1][m];
    }
    return;
  }
#pragma unroll 1
  for (int q = 0; q < 2; ++q) {
    float2 x[1][V];
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const int c = t + T * m;
      const float kx = wn<N>(c);
      const float k2 = kx * kx + ky * ky;
      const float inv = k2 > 0.f ? __frcp_rn(k2) : 0.f;
      const float2 w = own1[PL::pad(c)];
      if (q == 0) {
        const float fa = (1.f - ky * inv) * inv_n2;     // w + i u_hat = w (1 - ky/k2)
        x[0][m] = make_float2(w.x * fa, w.y * fa);
      } else {
        const float fb = kx * inv * inv_n2;              // v_hat = -i kx w / k2
        x[0][m] = make_float2(w.y * fb, -w.x * fb);
      }
    }
    float2* const xb[1] = {own0};
    fft_lines<N, V, +1, 1>(x, xb, t, a.tw, CtaSync{});
    float2* const dst = q == 0 ? a.pa : a.pb;
#pragma unroll
    for (int m = 0; m < V; ++m) dst[rbase + t + T * m] = x[0][m];
  }
}

// initialise the tile barrier of a spectral-row CTA (all threads call; one initialises)
template <int N, class TU = Tune<N>> __device__ __forceinline__ uint64_t* spec_barrier_init(float2* smem) {
  uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(smem) + TU::B_BAR_OFF);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  return bar;
}

template <int N, int MODE, bool PTR, class TU = Tune<N>>
__global__ void __launch_bounds__(TU::B_THREADS, TU::B_MINB) k_spec_rows(SpecArgs a) {
  extern __shared__ __align__(16) float2 smem[];
  uint64_t* bar = spec_barrier_init<N, TU>(smem);
  spec_rows_tile<N, MODE, PTR, TU>(a, blockIdx.x, smem, bar, 0u);
}

// ---------------------------------------------------------------------------------------
// standalone 2D FFT passes (Fft2D.run, fft.js:81-92): rows (x) then columns (y).
// SIGN -1 forward unscaled; +1 inverse scaled 1/N per pass (fft.js:58-59).
template <int N, int SIGN>
__global__ void __launch_bounds__(Tune<N>::B_THREADS) k_fft_rows(float2* data, const float2* tw) {
  using TU = Tune<N>;
  constexpr int V = TU::V, T = TU::T;
  extern __shared__ float2 smem[];
  const int t = threadIdx.x % T, slot = threadIdx.x / T;
  const size_t base = (size_t)(blockIdx.x * TU::B_ROWS + slot) * N;
  float2 x[1][V];
#pragma unroll
  for (int m = 0; m < V; ++m) x[0][m] = data[base + t + T * m];
  float2* const b[1] = {smem + slot * TU::B_LDS};
  fft_lines<N, V, SIGN, 1>(x, b, t, tw, CtaSync{});
  constexpr float sc = SIGN > 0 ? 1.0f / N : 1.0f;
#pragma unroll
  for (int m = 0; m < V; ++m) data[base + t + T * m] = cscale(x[0][m], sc);
}

template <int N, int SIGN>
__global__ void __launch_bounds__(Tune<N>::A_THREADS) k_fft_cols(float2* data, const float2* tw) {
  using TU = Tune<N>;
  constexpr int V = TU::V, T = TU::T, GA = TU::GA;
  extern __shared__ float2 smem[];
  const int g = threadIdx.x % GA, t = threadIdx.x / GA;
  const int col = blockIdx.x * GA + g;
  float2 x[1][V];
#pragma unroll
  for (int m = 0; m < V; ++m) x[0][m] = data[(size_t)(t + T * m) * N + col];
  float2* const b[1] = {smem + g * TU::A_LDS};
  fft_lines<N, V, SIGN, 1>(x, b, t, tw, CtaSync{});
  constexpr float sc = SIGN > 0 ? 1.0f / N : 1.0f;
#pragma unroll
  for (int m = 0; m < V; ++m) data[(size_t)(t + T * m) * N + col] = cscale(x[0][m], sc);
}

// ---------------------------------------------------------------------------------------
// elementwise reference stages (one thread per cell, any N)
static __global__ void k_velocity_pack(const float2* __restrict__ w, float2* pa, float2* pb, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  const float kx = wn_rt(idx & (n - 1), n), ky = wn_rt(idx / n, n);
  const float k2 = kx * kx + ky * ky;
  const float inv = k2 > 0.f ? 1.f / k2 : 0.f;
  const float2 ww = w[idx];
  const float2 iw = make_float2(-ww.y, ww.x);
  const float2 uh = cscale(iw, ky * inv);
  const float2 vh = cscale(iw, -kx * inv);
  pa[idx] = make_float2(ww.x - uh.y, ww.y + uh.x);   // w + i*uh (solver.wgsl:38)
  pb[idx] = vh;
}

static __global__ void k_nl_pack(const float2* __restrict__ pa, const float2* __restrict__ pb, float2* physz,
                          float2* vel, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  const float2 a = pa[idx];
  const float om = a.x, u = a.y, v = pb[idx].x;
  physz[idx] = make_float2(u * om, v * om);
  vel[idx] = make_float2(u, v);
}

static __global__ void k_assemble(const float2* __restrict__ physz, const float2* __restrict__ fhat,
                           const float* __restrict__ dtbuf, const DevParams* __restrict__ params,
                           float2* rhs, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  const DevParams& P = *params;
  const int col = idx & (n - 1), row = idx / n;
  const float kx = wn_rt(col, n), ky = wn_rt(row, n);
  const float k2 = kx * kx + ky * ky;
  const float2 zk = physz[idx];
  const float2 zm = cconj(physz[((n - row) & (n - 1)) * n + ((n - col) & (n - 1))]);
  const float2 q1 = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
  const float2 dd = csub(zk, zm);
  const float2 q2 = make_float2(0.5f * dd.y, -0.5f * dd.x);
  const float2 nhat = make_float2(-(kx * q1.y) - ky * q2.y, kx * q1.x + ky * q2.x);
  const float mask = (fabsf(kx) < P.kcut && fabsf(ky) < P.kcut) ? 1.f : 0.f;
  float2 f = cscale(csub(fhat ? fhat[idx] : make_float2(0.f, 0.f), nhat), mask);   // no pointer force: nullptr
  if (P.force_amp > 0.f && mask > 0.f && k2 > 0.f)
    f = cadd(f, stochastic_term(P, n, row, col, kx, ky, k2, dtbuf[0]));
  rhs[idx] = f;
}

// the per-substep stepIndex latch (S2D_STEP_RELATCH) as a launch of its own, for steps
// whose first kernel is not the fused column kernel that otherwise performs it
static __global__ void k_latch_step(DevParams* params, uint32_t* counter) {
  const uint32_t k = *counter;
  params->step_index = k;
  *counter = k + 1u;
}

template <int S>
__global__ void k_rk3(const float2* __restrict__ w0, const float2* __restrict__ wcur, float2* wout,
                      const float2* __restrict__ rhs, const float* __restrict__ dtbuf,
                      const DevParams* __restrict__ params, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n) return;
  const float kx = wn_rt(idx & (n - 1), n), ky = wn_rt(idx / n, n);
  const float k2 = kx * kx + ky * ky;
  if (k2 == 0.f) {
    wout[idx] = make_float2(0.f, 0.f);
    return;
  }
  const float dt = dtbuf[0];
  wout[idx] = rk_update<S>(half_factor_m1(*params, kx, k2, dt), w0[idx], wcur[idx], rhs[idx], dt);
}

}  // namespace s2d
