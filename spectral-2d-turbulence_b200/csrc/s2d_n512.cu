// Kernel instantiations for N = 512 (one translation unit per grid size so the
// per-size template expansions compile in parallel).
#include "s2d_ops.cuh"

namespace s2d {
const NOps* ops_n512() {
  // extra stage shapes the autotuner may pick (radix-8 line passes, more resident CTAs)
  static const NOps o = OpsImpl<512>::make({PhysImpl<512, Tune<512, 8>>::make("V=8")},
                                      {SpecImpl<512, Tune<512, 8>>::make("V=8"),
                                       SpecImpl<512, Tune<512, 8, 0, 6>>::make("V=8, 6 CTAs/SM"),
                                       SpecImpl<512, Tune<512, 8, 0, 6, true>>::make("V=8, 6 CTAs/SM, staged rows")});
  return &o;
}
}  // namespace s2d
