// Kernel instantiations for N = 1024 (one translation unit per grid size so the
// per-size template expansions compile in parallel).
#include "s2d_ops.cuh"

namespace s2d {
const NOps* ops_n1024() {
  static const NOps o = OpsImpl<1024>::make();
  return &o;
}
}  // namespace s2d
