// s2d_ops.cuh -- per-grid-size launch tables for the templated kernels.
#pragma once
#include <cuda_runtime.h>
#include "s2d_kernels.cuh"

namespace s2d {

struct NOps {
  int n;
  int a_grid, a_threads, b_grid, b_threads;
  size_t a_smem, b_smem, rows_smem, cols_smem;
  cudaError_t (*set_attrs)();
  void (*phys_cols)(int mode, const PhysArgs& a, cudaStream_t st);
  void (*spec_rows)(int mode, bool ptr, const SpecArgs& a, cudaStream_t st);
  void (*fft_rows)(int sign, float2* data, const float2* tw, cudaStream_t st);
  void (*fft_cols)(int sign, float2* data, const float2* tw, cudaStream_t st);
};

template <class K> inline cudaError_t set_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int N> struct OpsImpl {
  using TU = Tune<N>;
  static cudaError_t set_attrs() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) { if (r != cudaSuccess && e == cudaSuccess) e = r; };
    chk(set_smem(k_phys_cols<N, 0>, TU::A_SMEM));
    chk(set_smem(k_phys_cols<N, 1>, TU::A_SMEM));
    chk(set_smem(k_phys_cols<N, 2>, TU::A_SMEM));
    chk(set_smem(k_spec_rows<N, -1, false>, TU::B_SMEM_TOTAL));
    chk(set_smem(k_spec_rows<N, 0, false>, TU::B_SMEM_TOTAL));
    chk(set_smem(k_spec_rows<N, 1, false>, TU::B_SMEM_TOTAL));
    chk(set_smem(k_spec_rows<N, 2, false>, TU::B_SMEM_TOTAL));
    chk(set_smem(k_spec_rows<N, 0, true>, TU::B_SMEM_TOTAL));
    chk(set_smem(k_spec_rows<N, 1, true>, TU::B_SMEM_TOTAL));
    chk(set_smem(k_spec_rows<N, 2, true>, TU::B_SMEM_TOTAL));
    chk(set_smem(k_fft_rows<N, -1>, TU::ROWS_SMEM));
    chk(set_smem(k_fft_rows<N, +1>, TU::ROWS_SMEM));
    chk(set_smem(k_fft_cols<N, -1>, TU::COLS_SMEM));
    chk(set_smem(k_fft_cols<N, +1>, TU::COLS_SMEM));
    return e;
  }
  static void phys_cols(int mode, const PhysArgs& a, cudaStream_t st) {
    const dim3 g(TU::A_GRID), b(TU::A_THREADS);
    if (mode == 0) k_phys_cols<N, 0><<<g, b, TU::A_SMEM, st>>>(a);
    else if (mode == 1) k_phys_cols<N, 1><<<g, b, TU::A_SMEM, st>>>(a);
    else k_phys_cols<N, 2><<<g, b, TU::A_SMEM, st>>>(a);
  }
  static void spec_rows(int mode, bool ptr, const SpecArgs& a, cudaStream_t st) {
    const dim3 g(TU::B_GRID), b(TU::B_THREADS);
    switch (mode) {
      case -1: k_spec_rows<N, -1, false><<<g, b, TU::B_SMEM_TOTAL, st>>>(a); break;
      case 0:
        if (ptr) k_spec_rows<N, 0, true><<<g, b, TU::B_SMEM_TOTAL, st>>>(a);
        else k_spec_rows<N, 0, false><<<g, b, TU::B_SMEM_TOTAL, st>>>(a);
        break;
      case 1:
        if (ptr) k_spec_rows<N, 1, true><<<g, b, TU::B_SMEM_TOTAL, st>>>(a);
        else k_spec_rows<N, 1, false><<<g, b, TU::B_SMEM_TOTAL, st>>>(a);
        break;
      default:
        if (ptr) k_spec_rows<N, 2, true><<<g, b, TU::B_SMEM_TOTAL, st>>>(a);
        else k_spec_rows<N, 2, false><<<g, b, TU::B_SMEM_TOTAL, st>>>(a);
        break;
    }
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
  static NOps make() {
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
    o.set_attrs = &set_attrs;
    o.phys_cols = &phys_cols;
    o.spec_rows = &spec_rows;
    o.fft_rows = &fft_rows;
    o.fft_cols = &fft_cols;
    return o;
  }
};

}  // namespace s2d
