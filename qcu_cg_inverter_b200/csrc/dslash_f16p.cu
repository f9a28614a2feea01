// Stencil kernel instantiations for batched launches of OP_HALF_FAST: two
// right-hand sides per thread (qcu_dslash_pair.cuh; same storage formats).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f16p(bool dag, int epi, int fin) {
  return dag ? pick<OP_HALF_FAST_2, true>(epi, fin) : pick<OP_HALF_FAST_2, false>(epi, fin);
}
}  // namespace qcu
