// Stencil kernel instantiations for PREC_SINGLE storage (split per precision so the
// variants compile in parallel).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f32(bool dag, int epi, int fin) {
  return dag ? pick<PREC_SINGLE, true>(epi, fin) : pick<PREC_SINGLE, false>(epi, fin);
}
}  // namespace qcu
