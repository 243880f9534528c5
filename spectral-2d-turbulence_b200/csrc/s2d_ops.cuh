// s2d_ops.cuh -- per-grid-size launch tables for the templated kernels.
//
// Each grid size registers one or more launch shapes (Tune<N, V, minBlocks>) of the two
// stage kernels; index 0 is the default shape Tune<N>.  The autotuner (s2d_autotune)
// times the registered shapes on the solver's own state and keeps the fastest column
// and row variants.
#pragma once
#include <cuda_runtime.h>
#include "s2d_kernels.cuh"

namespace s2d {

// Launch with the given dynamic shared memory
template <class K> inline cudaError_t set_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

struct PhysVariant {
  const char* name;
  cudaError_t (*set_attrs)();
  void (*run)(int mode, const PhysArgs& a, cudaStream_t st);
};
struct SpecVariant {
  const char* name;
  cudaError_t (*set_attrs)();
  void (*run)(int mode, bool ptr, const SpecArgs& a, cudaStream_t st);
};
constexpr int kMaxVariants = 4;

struct NOps {
  int n;
  // the default shape (standalone FFT passes, ensembles, tables)
  int a_grid, a_threads, b_grid, b_threads;
  size_t a_smem, b_smem, rows_smem, cols_smem;
  cudaError_t (*set_attrs)();   // FFT passes and every registered stage variant
  void (*fft_rows)(int sign, float2* data, const float2* tw, cudaStream_t st);
  void (*fft_cols)(int sign, float2* data, const float2* tw, cudaStream_t st);
  int n_phys = 0, n_spec = 0;
  PhysVariant phys[kMaxVariants];
  SpecVariant spec[kMaxVariants];
};

// ---------------------------------------------------------------- column-stage variant
template <int N, class TU> struct PhysImpl {
  static cudaError_t set_attrs() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) { if (r != cudaSuccess && e == cudaSuccess) e = r; };
    chk(set_smem(k_phys_cols<N, 0, TU>, TU::A_SMEM));
    chk(set_smem(k_phys_cols<N, 1, TU>, TU::A_SMEM));
    chk(set_smem(k_phys_cols<N, 2, TU>, TU::A_SMEM));
    return e;
  }
  static void run(int mode, const PhysArgs& a, cudaStream_t st) {
    const dim3 g(TU::A_GRID), b(TU::A_THREADS);
    if (mode == 0) k_phys_cols<N, 0, TU><<<g, b, TU::A_SMEM, st>>>(a);
    else if (mode == 1) k_phys_cols<N, 1, TU><<<g, b, TU::A_SMEM, st>>>(a);
    else k_phys_cols<N, 2, TU><<<g, b, TU::A_SMEM, st>>>(a);
  }
  static PhysVariant make(const char* name) { return PhysVariant{name, &set_attrs, &run}; }
};

// ---------------------------------------------------------------- row-stage variant
template <int N, class TU> struct SpecImpl {
  template <int MODE, bool PTR> static cudaError_t attr() {
    return set_smem(k_spec_rows<N, MODE, PTR, TU>, spec_smem<TU, MODE, PTR>());
  }
  static cudaError_t set_attrs() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) { if (r != cudaSuccess && e == cudaSuccess) e = r; };
    chk(attr<-1, false>());
    chk(attr<0, false>());
    chk(attr<1, false>());
    chk(attr<2, false>());
    chk(attr<0, true>());
    chk(attr<1, true>());
    chk(attr<2, true>());
    return e;
  }
  template <int MODE, bool PTR> static void launch(const SpecArgs& a, cudaStream_t st) {
    k_spec_rows<N, MODE, PTR, TU><<<dim3(TU::B_GRID), dim3(TU::B_THREADS), spec_smem<TU, MODE, PTR>(), st>>>(a);
  }
  static void run(int mode, bool ptr, const SpecArgs& a, cudaStream_t st) {
    switch (mode) {
      case -1: launch<-1, false>(a, st); break;
      case 0: ptr ? launch<0, true>(a, st) : launch<0, false>(a, st); break;
      case 1: ptr ? launch<1, true>(a, st) : launch<1, false>(a, st); break;
      default: ptr ? launch<2, true>(a, st) : launch<2, false>(a, st); break;
    }
  }
  static SpecVariant make(const char* name) { return SpecVariant{name, &set_attrs, &run}; }
};

// ---------------------------------------------------------------- per-size table
template <int N> struct OpsImpl {
  using TU = Tune<N>;
  static cudaError_t fft_attrs() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) { if (r != cudaSuccess && e == cudaSuccess) e = r; };
    chk(set_smem(k_fft_rows<N, -1>, TU::ROWS_SMEM));
    chk(set_smem(k_fft_rows<N, +1>, TU::ROWS_SMEM));
    chk(set_smem(k_fft_cols<N, -1>, TU::COLS_SMEM));
    chk(set_smem(k_fft_cols<N, +1>, TU::COLS_SMEM));
    return e;
  }
  static void fft_rows(int sign, float2* d, const float2* tw, cudaStream_t st) {
    const dim3 g(N / TU::B_ROWS), b(TU::B_THREADS);
    if (sign < 0) k_fft_rows<N, -1><<<g, b, TU::ROWS_SMEM, st>>>(d, tw);
    else k_fft_rows<N, +1><<<g, b, TU::ROWS_SMEM, st>>>(d, tw);
  }
  static void fft_cols(int sign, float2* d, const float2* tw, cudaStream_t st) {
    const dim3 g(N / TU::GA), b(TU::A_THREADS);
    if (sign < 0) k_fft_cols<N, -1><<<g, b, TU::COLS_SMEM, st>>>(d, tw);
    else k_fft_cols<N, +1><<<g, b, TU::COLS_SMEM, st>>>(d, tw);
  }
  // the default shape, plus the extra shapes given as (name, variant) lists
  static NOps make(std::initializer_list<PhysVariant> extra_phys = {},
                   std::initializer_list<SpecVariant> extra_spec = {}) {
    NOps o;
    o.n = N;
    o.a_grid = TU::A_GRID;
    o.a_threads = TU::A_THREADS;
    o.b_grid = TU::B_GRID;
    o.b_threads = TU::B_THREADS;
    o.a_smem = TU::A_SMEM;
    o.b_smem = TU::B_SMEM_TOTAL;
    o.rows_smem = TU::ROWS_SMEM;
    o.cols_smem = TU::COLS_SMEM;
    o.set_attrs = &fft_attrs;
    o.fft_rows = &fft_rows;
    o.fft_cols = &fft_cols;
    o.phys[o.n_phys++] = PhysImpl<N, TU>::make("V=16");
    o.spec[o.n_spec++] = SpecImpl<N, TU>::make("V=16");
    for (const PhysVariant& v : extra_phys)
      if (o.n_phys < kMaxVariants) o.phys[o.n_phys++] = v;
    for (const SpecVariant& v : extra_spec)
      if (o.n_spec < kMaxVariants) o.spec[o.n_spec++] = v;
    return o;
  }
};

// every attribute a size needs: FFT passes and all its stage variants
inline cudaError_t set_all_attrs(const NOps& o) {
  cudaError_t e = o.set_attrs();
  for (int i = 0; i < o.n_phys && e == cudaSuccess; ++i) e = o.phys[i].set_attrs();
  for (int i = 0; i < o.n_spec && e == cudaSuccess; ++i) e = o.spec[i].set_attrs();
  return e;
}

}  // namespace s2d
