// Deterministic single-pass reductions.
//
// Kernels run with a 2-D thread block: threadIdx.x = right-hand side within the
// block's RHS tile (Rb lanes), threadIdx.y = site. Each block reduces its
// per-RHS values with warp shuffles (over the site lanes only) and shared
// memory, writes one partial per (rhs, quantity), and the last block to finish
// (atomic ticket) sums the partials in a fixed order and calls a finishing
// functor with the totals. The result therefore depends only on the launch
// shape, never on timing. Partials and tickets live in caller-provided scratch
// memory; the last block re-arms the ticket to 0.
#pragma once
#include "qcu_common.cuh"

namespace qcu {

struct ReduceArgs {
  double* partial;      // [nrhs*NR][gridDim.x] doubles
  unsigned* ticket;     // one counter, 0 on entry
  double* result;       // [nrhs*NR] totals (written by the last block)
  void* state;          // passed to the finishing functor
};

// No finishing step: totals are left in result[].
struct FinNone {
  static QCU_D void apply(const double*, int, int, void*) {}
};

// every reducing kernel is launched with at most 256 threads (its
// __launch_bounds__), so a block has at most 8 warps; the shared array is sized
// for that (smaller arrays leave more of the SM's memory to the L1 cache)
constexpr int kMaxWarps = 8;

// The block's place in a (site tile, RHS tile) launch grid: by default
// blockIdx.x / gridDim.x over site tiles and blockIdx.y over RHS tiles.
// nblocks: the blocks that take part in the reduction (the last of them to
// finish sums the partials); more than the launch's own when several launches
// over disjoint sites share one reduction.
struct TileCoord {
  int site, nsite, rhs;
  unsigned nblocks;
  static QCU_D TileCoord from_grid() {
    return TileCoord{(int)blockIdx.x, (int)gridDim.x, (int)blockIdx.y, gridDim.x * gridDim.y};
  }
};

// vals: NR values for each of the RL right-hand sides of this thread (RHS
// (t.rhs*Rb + threadIdx.x)*RL + j holds vals[j*NR .. j*NR+NR-1]; zero for idle
// threads). Every thread of the block must call this.
template <int NR, class Fin, int RL = 1>
QCU_D void block_reduce_finish(double vals[NR * RL], int nrhs, const ReduceArgs& red,
                               const TileCoord t = TileCoord::from_grid()) {
  __shared__ double sm[kMaxWarps][NR * RL * 32];
  __shared__ bool am_last;
  const int Rb = blockDim.x;
  const int tid = threadIdx.y * Rb + threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int nthreads = Rb * blockDim.y;
  const int nwarps = (nthreads + 31) >> 5;
  // reduce over the site lanes of the warp (lanes that share threadIdx.x)
#pragma unroll
  for (int k = 0; k < NR * RL; k++)
    for (int off = 16; off >= Rb; off >>= 1) vals[k] += __shfl_xor_sync(0xffffffffu, vals[k], off);
  if (lane < Rb)
    for (int k = 0; k < NR * RL; k++) sm[warp][k * 32 + lane] = vals[k];
  __syncthreads();
  if (threadIdx.y == 0) {
    for (int j = 0; j < RL; j++) {
      const int r = (t.rhs * Rb + threadIdx.x) * RL + j;
      if (r < nrhs) {
        for (int k = 0; k < NR; k++) {
          double acc = 0.0;
          for (int w = 0; w < nwarps; w++) acc += sm[w][(j * NR + k) * 32 + threadIdx.x];
          red.partial[(size_t)(r * NR + k) * t.nsite + t.site] = acc;
        }
      }
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    const unsigned total = t.nblocks;
    unsigned t = atomicAdd(red.ticket, 1u);
    am_last = (t == total - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  // last block: one warp per (rhs, quantity), lanes stride over the blocks
  const int nq = nrhs * NR;
  for (int q = warp; q < nq; q += nwarps) {
    double acc = 0.0;
    const volatile double* p = red.partial + (size_t)q * t.nsite;
    for (int b = lane; b < t.nsite; b += 32) acc += p[b];
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) red.result[q] = acc;
  }
  __syncthreads();
  if (tid == 0) {
    Fin::apply(red.result, nrhs, NR, red.state);
    __threadfence();
    *red.ticket = 0u;
  }
}

}  // namespace qcu
