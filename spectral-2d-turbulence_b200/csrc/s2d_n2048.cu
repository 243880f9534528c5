// Kernel instantiations for N = 2048 (one translation unit per grid size so the
// per-size template expansions compile in parallel).
#include "s2d_ops.cuh"

namespace s2d {
const NOps* ops_n2048() {
  static const NOps o = OpsImpl<2048>::make();
  return &o;
}
}  // namespace s2d
