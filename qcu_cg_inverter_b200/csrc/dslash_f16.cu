// Stencil kernel instantiations for PREC_HALF storage (split per precision so the
// variants compile in parallel).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f16(bool dag, int epi, int fin) {
  return dag ? pick<PREC_HALF, true>(epi, fin) : pick<PREC_HALF, false>(epi, fin);
}
}  // namespace qcu
