// Launcher of the fused stencil kernels (instantiated per precision in
// dslash_f64.cu, dslash_f32.cu and dslash_f16.cu).
#include "qcu_kernels.cuh"

namespace qcu {

typedef void (*DslashKernelFn)(const DslashArgs);
DslashKernelFn pick_f64(bool dag, int epi, int fin);
DslashKernelFn pick_f32(bool dag, int epi, int fin);
DslashKernelFn pick_f16(bool dag, int epi, int fin);
DslashKernelFn pick_f16x(bool dag, int epi, int fin);
DslashKernelFn pick_f16x1(bool dag, int epi, int fin);

cudaError_t launch_dslash(int prec, bool dagger, int epi, int fin, const DslashArgs& a, LaunchShape sh,
                          cudaStream_t stream) {
  DslashKernelFn fn = nullptr;
  switch (prec) {
    case PREC_DOUBLE: fn = pick_f64(dagger, epi, fin); break;
    case PREC_SINGLE: fn = pick_f32(dagger, epi, fin); break;
    case PREC_HALF: fn = pick_f16(dagger, epi, fin); break;
    case OP_HALF_FAST: fn = a.nrhs == 1 ? pick_f16x1(dagger, epi, fin) : pick_f16x(dagger, epi, fin); break;
    default: break;
  }
  if (!fn) return cudaErrorInvalidValue;
  if (sh.Rb < 1 || sh.Rb > 32 || (32 % sh.Rb) != 0 || (sh.Rb * sh.Sb) % 32 != 0 || sh.Rb * sh.Sb > 256)
    return cudaErrorInvalidConfiguration;
  dim3 block(sh.Rb, sh.Sb);
  dim3 grid(grid_x(a.g.Vh, sh.Sb), (a.nrhs + sh.Rb - 1) / sh.Rb);
  fn<<<grid, block, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace qcu
