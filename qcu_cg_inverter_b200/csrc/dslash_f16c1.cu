// Stencil kernel instantiations for single-RHS launches of OP_HALF (16-bit
// spinors, 16-bit 12-real links, 16-bit clover; block-paired epilogues).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f16c1(bool dag, int epi, int fin) {
  return dag ? pick<OP_HALF_1, true>(epi, fin) : pick<OP_HALF_1, false>(epi, fin);
}
}  // namespace qcu
