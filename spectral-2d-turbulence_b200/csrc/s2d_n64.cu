// Kernel instantiations for N = 64 (one translation unit per grid size so the
// per-size template expansions compile in parallel).
#include "s2d_ops.cuh"

namespace s2d {
const NOps* ops_n64() {
  static const NOps o = OpsImpl<64>::make();
  return &o;
}
}  // namespace s2d
