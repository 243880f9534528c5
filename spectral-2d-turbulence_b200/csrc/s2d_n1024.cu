// Kernel instantiations for N = 1024 (one translation unit per grid size so the
// per-size template expansions compile in parallel).
#include "s2d_ops.cuh"

namespace s2d {
const NOps* ops_n1024() {
  // extra stage shapes the autotuner may pick (radix-8 line passes, more resident CTAs)
  static const NOps o = OpsImpl<1024>::make({PhysImpl<1024, Tune<1024, 8, 2>>::make("V=8, 2 CTAs/SM")},
                                       {SpecImpl<1024, Tune<1024, 8, 0, 4>>::make("V=8, 4 CTAs/SM"),
                                        SpecImpl<1024, Tune<1024, 8, 0, 3>>::make("V=8, 3 CTAs/SM"),
                                        SpecImpl<1024, Tune<1024, 8, 0, 3, false, true>>::make(
                                            "V=8, 3 CTAs/SM, paired inverse transforms")});
  return &o;
}
}  // namespace s2d
