// Stencil kernel instantiations for PREC_DOUBLE storage (split per precision so the
// variants compile in parallel).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f64(bool dag, int epi, int fin) {
  return dag ? pick<PREC_DOUBLE, true>(epi, fin) : pick<PREC_DOUBLE, false>(epi, fin);
}
}  // namespace qcu
