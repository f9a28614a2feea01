// Stencil kernel instantiations for batched launches of OP_HALF_FAST: two
// right-hand sides per thread, with the t neighbours' words staged in shared
// memory (qcu_dslash_pair.cuh; same storage formats).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f16pt(bool dag, int epi, int fin) {
  return dag ? pick<OP_HALF_FAST_2T, true>(epi, fin) : pick<OP_HALF_FAST_2T, false>(epi, fin);
}
}  // namespace qcu
