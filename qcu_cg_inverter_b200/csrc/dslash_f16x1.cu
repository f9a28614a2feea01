// Stencil kernel instantiations for single-RHS launches of OP_HALF_FAST
// (block-paired epilogues; same storage formats).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f16x1(bool dag, int epi, int fin) {
  return dag ? pick<OP_HALF_FAST_1, true>(epi, fin) : pick<OP_HALF_FAST_1, false>(epi, fin);
}
}  // namespace qcu
