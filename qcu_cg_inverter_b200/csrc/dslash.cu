// Launcher of the fused stencil kernels (instantiated per precision in
// dslash_f64.cu, dslash_f32.cu and dslash_f16.cu).
#include <stdlib.h>

#include "qcu_cg_state.cuh"
#include "qcu_kernels.cuh"

namespace qcu {

typedef void (*DslashKernelFn)(const DslashArgs);
DslashKernelFn pick_f64(bool dag, int epi, int fin);
DslashKernelFn pick_f32(bool dag, int epi, int fin);
DslashKernelFn pick_f16(bool dag, int epi, int fin);
DslashKernelFn pick_f16x(bool dag, int epi, int fin);
DslashKernelFn pick_f16x1(bool dag, int epi, int fin);
DslashKernelFn pick_f16p(bool dag, int epi, int fin);
DslashKernelFn pick_f16pt(bool dag, int epi, int fin);
DslashKernelFn pick_f16pz(bool dag, int epi, int fin);
DslashKernelFn pick_f64b(bool dag, int epi, int fin);
DslashKernelFn pick_f16c1(bool dag, int epi, int fin);

// Batched FP64 launches on their own kernel family (OP_DOUBLE_BATCH: capped,
// row-at-a-time reconstruction) (1) or on the single-RHS one (0).
#ifndef QCU_F64_BATCH
#define QCU_F64_BATCH 1
#endif

// Batched launches of the fast 16-bit operator on the RHS-paired kernels (1)
// or on one RHS per thread (0).
#ifndef QCU_RHS_PAIRS
#define QCU_RHS_PAIRS 1
#endif
// The CG update stencil (EPI_CGXR: hop, xpay, x and r update) stays on one
// RHS per thread unless this is 1. Measured in the 48-RHS 24^3x48 solve with
// FP32 accumulators: 0.519 s with it on one RHS per thread, 0.528 s paired
// (loads grouped by three chunks), 0.546 s paired with one chunk at a time.
#ifndef QCU_PAIR_CGXR
#define QCU_PAIR_CGXR 0
#endif

// Single-RHS launches of the compact 16-bit operator (OP_HALF) on their own
// kernel family (OP_HALF_1: paired decode, block-paired epilogues) (1) or on
// the generic one (0).
#ifndef QCU_COMPACT_1RHS
#define QCU_COMPACT_1RHS 1
#endif

// Batched launches on a one-dimensional grid with the RHS tiles of each site
// tile adjacent (1), or on the (site tile, RHS tile) grid (0). Measured on
// B200, 24^3x48 with 48 RHS (6 RHS tiles of 8): the fused CG stencil K2 2167
// -> 1967 us (DRAM reads 3.93 -> 3.22 GB: the links and clover of a site tile
// come from DRAM once instead of once per RHS tile), the CG update stencil
// 1844 -> 1757 us, the 48-RHS batch 0.477 -> 0.455 s.
#ifndef QCU_SLAB_MINOR
#define QCU_SLAB_MINOR 1
#endif

static int g_pairs_override = -1;
void set_rhs_pairs_override(int v) { g_pairs_override = v; }

// RHS-paired launches with no neighbour words staged in shared memory (0),
// the t neighbours' (1) or the z and t neighbours' (2). The environment
// variable QCU_PAIR_STAGE overrides the built-in choice.
#ifndef QCU_PAIR_STAGE
#define QCU_PAIR_STAGE 0
#endif
static int g_stage_override = -1;
void set_pair_stage_override(int v) { g_stage_override = v; }
static int pair_stage() {
  static const int env = [] {
    const char* e = getenv("QCU_PAIR_STAGE");
    return e ? atoi(e) : -1;
  }();
  const int v = g_stage_override >= 0 ? g_stage_override : env >= 0 ? env : QCU_PAIR_STAGE;
  return v < 0 ? 0 : v > 2 ? 2 : v;
}
// Raises the dynamic shared memory limit of every staged kernel on the
// current device to the most any launch shape asks for (two staged
// directions, 256 thread slots); done when a context is created, so that no
// attribute changes while launches are captured into graphs.
cudaError_t prepare_staged_kernels() {
  const int bytes = staged_bytes(4, 8, 32);
  const int epis[] = {0, EPI_CPRE, EPI_XPAY, EPI_XPAY | EPI_CX, EPI_XPAY | EPI_CPOST, EPI_CPRE | EPI_XPAY,
                      EPI_CPRE | EPI_XPAY | EPI_NORM, EPI_CPRE | EPI_XPAY | EPI_OUT2,
                      EPI_CPRE | EPI_XPAY | EPI_OUT2 | EPI_NORM, EPI_XPAY | EPI_NORM, EPI_XPAY | EPI_CGXR};
  for (int dag = 0; dag < 2; dag++)
    for (int epi : epis)
      for (int fin : {(int)FIN_NONE, (int)FIN_CG_ALPHA, (int)FIN_CG_BETA}) {
        DslashKernelFn fn = pick_f16pz(dag != 0, epi, fin);
        if (!fn) continue;
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
      }
  return cudaSuccess;
}

cudaError_t launch_dslash(int prec, bool dagger, int epi, int fin, const DslashArgs& a, LaunchShape sh,
                          cudaStream_t stream, int* launched) {
  if (launched) *launched = 0;
  const bool pairs = g_pairs_override < 0 ? QCU_RHS_PAIRS != 0 : g_pairs_override != 0;
  const bool pair_cgxr = g_pairs_override < 0 ? QCU_PAIR_CGXR != 0 : g_pairs_override != 0;
  DslashKernelFn fn = nullptr;
  // RHS lanes per thread: the RHS-paired kernels take a block of Rb/2 x Sb
  // threads for the same Rb x Sb tile of (RHS, site)
  int per_thread = 1;
  int smem = 0;  // dynamic shared memory of the launch
  switch (prec) {
    case PREC_DOUBLE: fn = (QCU_F64_BATCH && a.nrhs > 1) ? pick_f64b(dagger, epi, fin) : pick_f64(dagger, epi, fin); break;
    case PREC_SINGLE: fn = pick_f32(dagger, epi, fin); break;
    case PREC_HALF: fn = (a.nrhs == 1 && QCU_COMPACT_1RHS) ? pick_f16c1(dagger, epi, fin) : pick_f16(dagger, epi, fin); break;
    case OP_HALF_FAST:
      if (a.nrhs == 1) {
        fn = pick_f16x1(dagger, epi, fin);
      } else if (pairs && sh.Rb >= 2 && (pair_cgxr || !(epi & EPI_CGXR))) {
        const int ns = pair_stage();
        fn = ns == 2 ? pick_f16pz(dagger, epi, fin) : ns == 1 ? pick_f16pt(dagger, epi, fin) : pick_f16p(dagger, epi, fin);
        smem = ns ? staged_bytes(2 * ns, sh.Rb, sh.Sb) : 0;
        per_thread = 2;
      } else {
        fn = pick_f16x(dagger, epi, fin);
      }
      break;
    default: break;
  }
  if (!fn) return cudaErrorInvalidValue;
  const int tx = sh.Rb / per_thread;
  if (sh.Rb < 1 || sh.Rb > 32 || (32 % sh.Rb) != 0 || (tx * sh.Sb) % 32 != 0 || sh.Rb * sh.Sb > 256)
    return cudaErrorInvalidConfiguration;
  dim3 block(tx, sh.Sb);
  const int nslab = (a.nrhs + sh.Rb - 1) / sh.Rb;
  const int nsites = (a.s_lim > 0 ? a.s_lim : a.g.Vh) - a.s_off;
  if (nsites <= 0) return cudaSuccess;

  // a reduction over this launch's site tiles alone, large enough to defer
  const int site_tiles = grid_x(nsites, sh.Sb);
  const bool reduces = (epi & (EPI_NORM | EPI_CGXR)) != 0;
  const bool defer = reduces && a.block_total == 0 && (size_t)a.nrhs * site_tiles >= kTwoLevelMin;
  DslashArgs b = a;
  b.red.deferred = defer ? 1 : 0;
  if (QCU_SLAB_MINOR && nslab > 1) {
    // the RHS tiles of one site tile run back to back, so its links and
    // clover are read from DRAM once and served from L2 to the others
    b.nslab = nslab;
    fn<<<dim3(site_tiles * nslab, 1), block, smem, stream>>>(b);
  } else {
    b.nslab = 0;
    fn<<<dim3(site_tiles, nslab), block, smem, stream>>>(b);
  }
  if (launched) *launched = 1;
  if (defer) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    switch (fin) {
      case FIN_CG_ALPHA: reduce_finish_kernel<FinCgAlpha><<<a.nrhs, 256, 0, stream>>>(b.red, site_tiles, a.nrhs, 1); break;
      case FIN_CG_BETA: reduce_finish_kernel<FinCgBeta><<<a.nrhs, 256, 0, stream>>>(b.red, site_tiles, a.nrhs, 1); break;
      default: reduce_finish_kernel<FinNone><<<a.nrhs, 256, 0, stream>>>(b.red, site_tiles, a.nrhs, 1); break;
    }
    if (launched) *launched = 2;
  }
  return cudaGetLastError();
}

}  // namespace qcu
