// Kernel argument structs and host launchers shared by the library's .cu files.
#pragma once
#include "qcu_common.cuh"
#include "qcu_fields.cuh"
#include "qcu_reduce.cuh"

namespace qcu {

// Epilogue flags of the fused stencil kernel. With h = D^(dag) in (the hop),
// C the clover field of the output parity, a the per-RHS coefficient and x the
// xpay input, the output is
//   EPI_CPRE           : out = C h
//   EPI_XPAY           : out = x + a h           (with EPI_CPRE: x + a C h)
//   EPI_XPAY|EPI_CX    : out = C x + a h
//   EPI_CPOST          : out = C (x + a h)       (needs EPI_XPAY)
//   EPI_OUT2           : also out2 = C out
//   EPI_NORM           : reduce |out|^2 per RHS (finishing functor FinId)
//   EPI_CGXR           : the CG update instead of a store (needs EPI_XPAY):
//                        xacc += alpha pvec, racc -= alpha out, reduce
//                        |racc|^2 (FinCgBeta); out never reaches memory
enum EpiFlags : int {
  EPI_CPRE = 1,
  EPI_XPAY = 2,
  EPI_CX = 4,
  EPI_CPOST = 8,
  EPI_OUT2 = 16,
  EPI_NORM = 32,
  EPI_CGXR = 64,
};

struct DslashArgs {
  Geom g;
  int parity;            // parity of the output sites
  int nrhs;
  CSpinorView in;        // parity 1-parity
  SpinorView out;
  CSpinorView x;         // xpay input, output parity
  SpinorView out2;
  const void* gauge;
  const void* clover;    // clover (or its inverse) field 0, both parities
  size_t clover_stride;  // bytes between resident clover fields
  const int* clover_idx; // per-RHS field index, nullptr -> field 0
  const double* coef;    // per-RHS a, nullptr -> coef0
  double coef0;
  double bc_t;
  const int* active;     // per-RHS mask, nullptr -> all active
  // RHS tiles per site tile when the grid is one-dimensional with the RHS
  // tiles of a site tile adjacent (blockIdx.x = site tile * nslab + RHS tile);
  // 0: two-dimensional grid (blockIdx.x site tile, blockIdx.y RHS tile)
  int nslab;
  // The launch covers sites [s_off, s_lim) (s_lim 0: the lattice's Vh). When
  // several launches over disjoint site ranges share one reduction, this
  // launch's site tiles are tiles tile_off ... of tile_total, and block_total
  // counts the blocks of all of them (0: this launch alone).
  int s_off, s_lim, tile_off, tile_total, block_total;
  ReduceArgs red;
  // EPI_CGXR: solution and residual in the accumulator precision (double for
  // FP64 spinors, else single), search direction in the spinor precision
  SpinorView xacc, racc;
  CSpinorView pvec;
  const double* alpha;
};

// Finishing functors available to fused reductions (see solver kernels).
// FIN_REL_CONT: marks the RHS that go on after a reliable update (the
// residual reduction of clover_res, or a one-block launch; never a stencil's)
enum FinId : int { FIN_NONE = 0, FIN_CG_ALPHA = 1, FIN_CG_BETA = 2, FIN_REL_CONT = 3 };

// shared-memory bytes of NT staged neighbours (16-bit words and norms of both
// lanes of every thread) of a block of RB/2 x SB threads (the RHS-paired
// kernels of qcu_dslash_pair.cuh)
QCU_HD constexpr int staged_bytes(int NT, int RB, int SB) { return NT * SB * RB * (3 * 16 + 4); }

// Launch configuration: block = (Rb rhs lanes, Sb site lanes).
struct LaunchShape {
  int Rb, Sb;
};

// `op` is an OpVariant (spinor / link / clover storage); the pointers in `a`
// must be fields of those formats.
// A reduction of at least kTwoLevelMin partials (and not shared with other
// launches) is deferred: the stencil only writes its partials and a finishing
// launch follows. *launched (if given) receives the number of kernels launched.
cudaError_t launch_dslash(int op, bool dagger, int epi, int fin, const DslashArgs& a, LaunchShape shape,
                          cudaStream_t stream, int* launched = nullptr);
// Test hook: batched launches of the fast 16-bit operator on the RHS-paired
// kernels for every epilogue (1), on one RHS per thread (0), or as built (-1).
void set_rhs_pairs_override(int v);
// Test hook: staged neighbours of the RHS-paired kernels (0 none, 1 t, 2 z
// and t, -1 as built)
void set_pair_stage_override(int v);
// the dynamic shared memory limit of the staged RHS-paired kernels, on the
// current device
cudaError_t prepare_staged_kernels();

// Number of blocks along x for a field of Vh sites.
inline int grid_x(int Vh, int Sb) { return (Vh + Sb - 1) / Sb; }

// The (site tile, RHS tile) of this block of a stencil launch.
QCU_D TileCoord stencil_tile(const DslashArgs& a) {
  TileCoord t = TileCoord::from_grid();
  if (a.nslab > 0) {
    const int st = blockIdx.x / a.nslab;
    t = TileCoord{st, (int)(gridDim.x / a.nslab), (int)(blockIdx.x - st * a.nslab), gridDim.x};
  }
  if (a.block_total > 0) {
    t.site += a.tile_off;
    t.nsite = a.tile_total;
    t.nblocks = (unsigned)a.block_total;
  }
  return t;
}
// first site of this block's tile and one past the launch's last site
QCU_D int stencil_site0(const DslashArgs& a, const TileCoord& t) {
  return a.s_off + (t.site - (a.block_total > 0 ? a.tile_off : 0)) * (int)blockDim.y;
}
QCU_D int stencil_slim(const DslashArgs& a) { return a.s_lim > 0 ? a.s_lim : a.g.Vh; }

}  // namespace qcu
