// Deterministic single-pass reductions.
//
// Kernels run with a 2-D thread block: threadIdx.x = right-hand side within the
// block's RHS tile (Rb lanes), threadIdx.y = site. Each block reduces its
// per-RHS values with warp shuffles (over the site lanes only) and shared
// memory and writes one partial per (rhs, quantity). The last block of each
// group of site tiles (atomic counters) sums the group's partials, and the
// last group sums the group sums, in a fixed order, and calls a finishing
// functor with the totals. The result therefore depends only on the launch
// shape, never on timing. Partials and counters live in caller-provided
// scratch memory; the blocks that finish re-arm the counters to 0.
#pragma once
#include "qcu_common.cuh"

namespace qcu {

struct ReduceArgs {
  double* partial;         // [nrhs*NR][site tiles] doubles
  unsigned* ticket;        // one counter, 0 on entry
  double* result;          // [nrhs*NR] totals (written by the last block)
  void* state;             // passed to the finishing functor
  double* partial2;        // [nrhs*NR][site-tile groups] doubles
  unsigned* group_ticket;  // [site-tile groups][RHS tiles] counters, 0 on entry
  // 1: the blocks only write their partials; a separate finishing launch
  // (reduce_finish_kernel) sums them and applies the functor
  int deferred;
};

// No finishing step: totals are left in result[].
struct FinNone {
  static QCU_D void apply(const double*, int, int, void*, int, int) {}
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

// Site tiles per group of the two-level finish: the last block of each group
// (per RHS tile) sums the group's partials into one second-level partial, and
// the last group to finish sums those and applies the functor.
constexpr int kReduceGroup = 128;
// Reductions of fewer partials (RHS x quantities x site tiles) than this keep
// the one-level finish: for them the second level's extra barrier, fence and
// counter on the last block's path cost more than its shorter sum (measured on
// B200: 16^3x32 single-RHS K2 14.6 us one-level, 16.4 us two-level)
constexpr size_t kTwoLevelMin = 4096;

// Sums p[b0], p[b0 + step], ... (indices below n) in that order. The loads
// bypass L1 (the partials were stored by other blocks of the launch) and eight
// are in flight at once; the adds keep the sequential order, so the total is
// the same as a plain loop's.
QCU_D double strided_sum(const double* p, int b0, int n, int step) {
  double acc = 0.0;
  int b = b0;
  for (; b + 7 * step < n; b += 8 * step) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = __ldcg(p + b + k * step);
#pragma unroll
    for (int k = 0; k < 8; k++) acc += v[k];
  }
  for (; b < n; b += step) acc += __ldcg(p + b);
  return acc;
}

// Adds one to a counter at GPU scope with acquire-release semantics. Called by
// thread 0 after a block barrier, the release covers every store the block
// made before the barrier (fences are cumulative), and the block that reads
// the final count sees all of the counted blocks' stores once it has passed
// its own barrier after this call. Cheaper than a sequentially consistent
// fence (__threadfence) followed by a relaxed atomic.
QCU_D unsigned ticket_arrive(unsigned* p) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
  return old;
}

// vals: NR values for each of the RL right-hand sides of this thread (RHS
// (t.rhs*Rb + threadIdx.x)*RL + j holds vals[j*NR .. j*NR+NR-1]; zero for idle
// threads). Every thread of the block must call this.
//
// Two-level finish (reductions of at least kTwoLevelMin partials): with one
// serial last block the final sum ran over every site tile (10368 per RHS at
// 24^3x48) on one SM while the GPU idled (measured on B200: the norm and its
// reduction cost the fused K2 0.33 of 1.95 ms with 48 RHS). Groups of
// kReduceGroup site tiles are summed by their last block as the launch runs;
// the last group then sums ceil(nsite / kReduceGroup) values per quantity
// (K2 with 48 RHS: 1.95 -> 1.79 ms). The order of every sum is fixed by the
// tile numbering, so the result still depends only on the launch shape.
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
  if (red.deferred) return;  // the finishing launch that follows sums the partials
  // The block counts once its partials are visible: after the barrier, thread
  // 0's fence orders every thread's stores before the counter (fences are
  // cumulative over the barrier, as in a release by one thread of the block).
  __syncthreads();
  if ((size_t)nrhs * NR * t.nsite < kTwoLevelMin) {
    // one level: the last block of the launch sums every partial
    if (tid == 0) am_last = (ticket_arrive(red.ticket) == t.nblocks - 1u);
    __syncthreads();
    if (!am_last) return;
    const int nq = nrhs * NR;
    for (int q = warp; q < nq; q += nwarps) {
      double acc = strided_sum(red.partial + (size_t)q * t.nsite, lane, t.nsite, 32);
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (lane == 0) red.result[q] = acc;
    }
    __syncthreads();
    Fin::apply(red.result, nrhs, NR, red.state, tid, nthreads);
    // the next launch that uses the counter sees the reset (launch boundary)
    if (tid == 0) *red.ticket = 0u;
    return;
  }
  // two levels: the block's arrival in its group
  const int ntiles = (int)(t.nblocks / (unsigned)t.nsite);  // RHS tiles
  const int ngroups = (t.nsite + kReduceGroup - 1) / kReduceGroup;
  const int g = t.site / kReduceGroup;
  const int g0 = g * kReduceGroup, g1 = min(g0 + kReduceGroup, t.nsite);
  if (tid == 0) am_last = (ticket_arrive(red.group_ticket + (size_t)g * ntiles + t.rhs) == (unsigned)(g1 - g0) - 1u);
  __syncthreads();
  if (!am_last) return;
  // last block of the group: its RHS tile's quantities, one warp each, lanes
  // over the group's site tiles
  {
    const int r0 = t.rhs * Rb * RL;
    const int nloc = max(0, min(Rb * RL, nrhs - r0)) * NR;
    for (int ql = warp; ql < nloc; ql += nwarps) {
      const int q = r0 * NR + ql;
      double acc = strided_sum(red.partial + (size_t)q * t.nsite, g0 + lane, g1, 32);
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (lane == 0) red.partial2[(size_t)q * ngroups + g] = acc;
    }
  }
  __syncthreads();
  if (tid == 0) {
    red.group_ticket[(size_t)g * ntiles + t.rhs] = 0u;  // every member has arrived
    // the release makes the group's sums visible before the group counts
    am_last = (ticket_arrive(red.ticket) == (unsigned)(ngroups * ntiles) - 1u);
  }
  __syncthreads();
  if (!am_last) return;
  // last group: one warp per (rhs, quantity), lanes over the groups
  const int nq = nrhs * NR;
  for (int q = warp; q < nq; q += nwarps) {
    double acc = strided_sum(red.partial2 + (size_t)q * ngroups, lane, ngroups, 32);
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) red.result[q] = acc;
  }
  __syncthreads();
  Fin::apply(red.result, nrhs, NR, red.state, tid, nthreads);
  if (tid == 0) *red.ticket = 0u;
}

// The finishing launch of a deferred reduction: block q sums quantity q's
// nsite partials (threads strided over them, then the warps in order), and the
// last block to finish applies the functor. A launch boundary makes the
// partials visible, so the reducing kernel's blocks end with their stores
// (measured on B200: the counters, fences and last-block sums inside the
// kernel had cost the fused K2 0.076 and K4 0.17 ms with 48 RHS at 24^3x48,
// and K2 14 us with one RHS at 32^3x64).
template <class Fin>
__global__ void __launch_bounds__(256) reduce_finish_kernel(ReduceArgs red, int nsite, int nrhs, int NR) {
  __shared__ double sm[kMaxWarps];
  __shared__ bool am_last;
  const int q = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  double acc = strided_sum(red.partial + (size_t)q * nsite, tid, nsite, blockDim.x);
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) sm[warp] = acc;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int w = 0; w < nwarps; w++) s += sm[w];
    red.result[q] = s;
    am_last = (ticket_arrive(red.ticket) == gridDim.x - 1u);
  }
  __syncthreads();
  if (!am_last) return;
  Fin::apply(red.result, nrhs, NR, red.state, tid, (int)blockDim.x);
  if (tid == 0) *red.ticket = 0u;
}

}  // namespace qcu
