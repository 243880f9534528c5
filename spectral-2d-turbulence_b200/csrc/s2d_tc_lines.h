// s2d_tc_lines.h -- host interface of the tensor-core line transforms for the grid sizes
// other than 1024 (s2d_tc_lines.cu).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace s2d {
namespace tc {
bool tc_lines_supported(int n);          // 256, 512, 2048, 4096
size_t tc_lines_table_bytes(int n);      // the per-solver DFT matrices (hi | lo planes)
cudaError_t tc_lines_attrs(int n, int bf16);
void tc_lines_tables(int n, int bf16, char* tab, const float2* tw, cudaStream_t st);
// 2D transform (rows, then columns) in place; sign -1 forward unscaled, +1 inverse / N per pass
void tc_lines_fft2(int n, int bf16, float2* buf, int sign, const char* tab, const float2* tw, int* err,
                   cudaStream_t st);
}  // namespace tc
}  // namespace s2d
