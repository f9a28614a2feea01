// The reference's storage shifts between its AoS layouts and its coalesced
// ("neo") SoA layouts (include/qcu_shift_storage.cuh:14-16,
// src/qcu_shift_storage.cu:75-195):
//   spinor, one parity block of nh = V/2 sites:
//     AoS [site][24 doubles]  <->  SoA [24][site]
//     (24 = spin*3 + colour components, re and im interleaved)
//   gauge, both parities of every direction:
//     AoS [dir][parity][site][9 complex]  ->  SoA [dir][parity][12][site]
//     (the first two rows of each link, re and im interleaved)
// The reference has no gauge shift back to AoS (its TO_NON_COALESCE branch
// does nothing); here it rebuilds the third row as conj(row0 x row1), the
// reference's reconstructSU3 (src/qcu_clover_dslash.cu:11-16).
//
// Each block transposes a tile of 128 sites through shared memory, so both
// the AoS side (24 or 18 consecutive doubles per site) and the SoA side (128
// consecutive doubles per component) are read and written in whole lines.
#include "qcu_context.h"

namespace qcu {

constexpr int kShiftTile = 128;

// spinor: to_soa = 1: [nh][24] -> [24][nh]; 0: [24][nh] -> [nh][24]
__global__ void __launch_bounds__(kShiftTile) shift_vector_kernel(double* __restrict__ dst,
                                                                  const double* __restrict__ src, int nh, int to_soa) {
  __shared__ double tile[kShiftTile * 24];
  const int s0 = blockIdx.x * kShiftTile;
  const int n = min(kShiftTile, nh - s0);
  if (to_soa) {
    for (int i = threadIdx.x; i < n * 24; i += kShiftTile) tile[i] = src[(size_t)s0 * 24 + i];
    __syncthreads();
    for (int i = threadIdx.x; i < kShiftTile * 24; i += kShiftTile) {
      const int c = i / kShiftTile, l = i - c * kShiftTile;
      if (l < n) dst[(size_t)c * nh + s0 + l] = tile[l * 24 + c];
    }
  } else {
    for (int i = threadIdx.x; i < kShiftTile * 24; i += kShiftTile) {
      const int c = i / kShiftTile, l = i - c * kShiftTile;
      if (l < n) tile[l * 24 + c] = src[(size_t)c * nh + s0 + l];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n * 24; i += kShiftTile) dst[(size_t)s0 * 24 + i] = tile[i];
  }
}

// gauge, one (direction, parity) block per blockIdx.y: to_soa = 1:
// [nh][18] -> [12][nh]; 0: [12][nh] -> [nh][18] with the third row rebuilt
__global__ void __launch_bounds__(kShiftTile) shift_gauge_kernel(double* __restrict__ dst,
                                                                 const double* __restrict__ src, int nh, int to_soa) {
  __shared__ double tile[kShiftTile * 18];
  const int s0 = blockIdx.x * kShiftTile;
  const int n = min(kShiftTile, nh - s0);
  const size_t mp = blockIdx.y;  // dir * 2 + parity
  if (to_soa) {
    const double* in = src + mp * nh * 18;
    double* out = dst + mp * nh * 12;
    for (int i = threadIdx.x; i < n * 18; i += kShiftTile) tile[i] = in[(size_t)s0 * 18 + i];
    __syncthreads();
    for (int i = threadIdx.x; i < kShiftTile * 12; i += kShiftTile) {
      const int c = i / kShiftTile, l = i - c * kShiftTile;
      if (l < n) out[(size_t)c * nh + s0 + l] = tile[l * 18 + c];
    }
  } else {
    const double* in = src + mp * nh * 12;
    double* out = dst + mp * nh * 18;
    for (int i = threadIdx.x; i < kShiftTile * 12; i += kShiftTile) {
      const int c = i / kShiftTile, l = i - c * kShiftTile;
      if (l < n) tile[l * 18 + c] = in[(size_t)c * nh + s0 + l];
    }
    __syncthreads();
    if ((int)threadIdx.x < n) {  // third row of this thread's link
      double* t = tile + threadIdx.x * 18;
      Link<double> U;
#pragma unroll
      for (int k = 0; k < 6; k++) U.u[k] = mk(t[2 * k], t[2 * k + 1]);
      su3_reconstruct(U);
#pragma unroll
      for (int k = 6; k < 9; k++) {
        t[2 * k] = U.u[k].re;
        t[2 * k + 1] = U.u[k].im;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n * 18; i += kShiftTile) out[(size_t)s0 * 18 + i] = tile[i];
  }
}

static int shift_check(void* dst, const void* src, int direction, int Lx, int Ly, int Lz, int Lt) {
  if (!dst || !src || (direction != 0 && direction != 1) || Lx <= 0 || Ly <= 0 || Lz <= 0 || Lt <= 0 || (Lx & 1) ||
      (long long)Lx * Ly * Lz * Lt / 2 > (1LL << 30) / 24) {
    set_error(QCU_ERR_INVALID_ARG, "bad storage-shift arguments");
    return QCU_ERR_INVALID_ARG;
  }
  if (!is_device_ptr(dst) || !is_device_ptr(src)) {
    set_error(QCU_ERR_INVALID_ARG, "storage shifts take device pointers");
    return QCU_ERR_INVALID_ARG;
  }
  return QCU_SUCCESS;
}

}  // namespace qcu

using namespace qcu;

extern "C" {

int qcuShiftVectorStorage(void* dst, const void* src, int direction, int Lx, int Ly, int Lz, int Lt) {
  clear_error();
  QCU_CHECK(shift_check(dst, src, direction, Lx, Ly, Lz, Lt));
  const int nh = Lx / 2 * Ly * Lz * Lt;
  shift_vector_kernel<<<(nh + kShiftTile - 1) / kShiftTile, kShiftTile>>>(
      static_cast<double*>(dst), static_cast<const double*>(src), nh, direction == 0 ? 1 : 0);
  QCU_CHECK_CUDA(cudaGetLastError());
  QCU_CHECK_CUDA(cudaStreamSynchronize(0));
  return QCU_SUCCESS;
}

int qcuShiftGaugeStorage(void* dst, const void* src, int direction, int Lx, int Ly, int Lz, int Lt) {
  clear_error();
  QCU_CHECK(shift_check(dst, src, direction, Lx, Ly, Lz, Lt));
  const int nh = Lx / 2 * Ly * Lz * Lt;
  dim3 grid((nh + kShiftTile - 1) / kShiftTile, 8);
  shift_gauge_kernel<<<grid, kShiftTile>>>(static_cast<double*>(dst), static_cast<const double*>(src), nh,
                                           direction == 0 ? 1 : 0);
  QCU_CHECK_CUDA(cudaGetLastError());
  QCU_CHECK_CUDA(cudaStreamSynchronize(0));
  return QCU_SUCCESS;
}

// The reference's C++ entry points under their C++ symbol names
// (include/qcu_shift_storage.cuh:14-16): void results, errors through
// qcu_last_error() instead of an exit.
void qcu_cxx_shiftVectorStorage(void* d, void* s, int dir, int Lx, int Ly, int Lz, int Lt) __asm__(
    "_Z18shiftVectorStoragePvS_iiiii");
void qcu_cxx_shiftVectorStorage(void* d, void* s, int dir, int Lx, int Ly, int Lz, int Lt) {
  (void)qcuShiftVectorStorage(d, s, dir, Lx, Ly, Lz, Lt);
}
void qcu_cxx_shiftGaugeStorage(void* d, void* s, int dir, int Lx, int Ly, int Lz, int Lt) __asm__(
    "_Z17shiftGaugeStoragePvS_iiiii");
void qcu_cxx_shiftGaugeStorage(void* d, void* s, int dir, int Lx, int Ly, int Lz, int Lt) {
  (void)qcuShiftGaugeStorage(d, s, dir, Lx, Ly, Lz, Lt);
}

}  // extern "C"
