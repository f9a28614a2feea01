// Stencil kernel instantiations for OP_HALF_FAST: 16-bit spinors, FP32
// 18-real links and FP32 clover (split per variant so they compile in parallel).
#include "qcu_dslash_impl.cuh"

namespace qcu {
DslashKernelFn pick_f16x(bool dag, int epi, int fin) {
  return dag ? pick<OP_HALF_FAST, true>(epi, fin) : pick<OP_HALF_FAST, false>(epi, fin);
}
}  // namespace qcu
