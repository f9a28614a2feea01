// Stencil kernel instantiations for batched launches on PREC_DOUBLE storage
// (OP_DOUBLE_BATCH: register cap and row-at-a-time reconstruction).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f64b(bool dag, int epi, int fin) {
  return dag ? pick<OP_DOUBLE_BATCH, true>(epi, fin) : pick<OP_DOUBLE_BATCH, false>(epi, fin);
}
}  // namespace qcu
