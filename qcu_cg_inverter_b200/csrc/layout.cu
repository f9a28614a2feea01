// Boundary layout conversions and seeded field generators.
//
// The reference's C interface exchanges fields in its AoS layouts
// (include/qcu_point.cuh:65-93): gauge [dir][parity][t][z][y][x/2][3][3] and
// spinors [parity][t][z][y][x/2][4][3], complex double. Its own ingest
// (loadQcuGauge, src/dslash.cu:27-35 -> shift_gauge_to_coalesed,
// src/qcu_shift_storage.cu:123-161) keeps the first two rows of every link as
// 12 reals; the conversions here do the same, into the site-blocked layout and
// any storage precision.
#include "qcu_fields.cuh"
#include "qcu_kernels.cuh"

namespace qcu {

// ---------------------------------------------------------------------------
// gauge: AoS FP64 -> internal (up to three precisions in one pass)
// ---------------------------------------------------------------------------
__global__ void gauge_aos_to_internal_kernel(Geom g, const double2* __restrict__ src, void* d64, void* d32, void* d16,
                                             void* d18) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;  // link index over [dir][parity][Vh]
  if (l >= 8 * g.Vh) return;
  const int mp = l / g.Vh, s = l - mp * g.Vh;
  const int mu = mp >> 1, parity = mp & 1;
  Link<double> U;
  const double2* p = src + (size_t)l * 9;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    double2 w = p[k];
    U.u[k] = mk(w.x, w.y);
  }
  if (d64) LinkIO<PREC_DOUBLE>::store(d64, g.Vh_pad, mu, parity, s, U);
  if (d32) LinkIO<PREC_SINGLE>::store(d32, g.Vh_pad, mu, parity, s, U);
  if (d16) LinkIO<PREC_HALF>::store(d16, g.Vh_pad, mu, parity, s, U);
  if (d18) {  // third row rebuilt in FP64 as everywhere else, then stored
    su3_reconstruct(U);
    LinkIO<LINK_SINGLE18>::store(d18, g.Vh_pad, mu, parity, s, U);
  }
}

cudaError_t launch_gauge_ingest(const Geom& g, const void* aos, void* d64, void* d32, void* d16, void* d18,
                                cudaStream_t st) {
  int n = 8 * g.Vh;
  gauge_aos_to_internal_kernel<<<(n + 127) / 128, 128, 0, st>>>(g, static_cast<const double2*>(aos), d64, d32, d16,
                                                                  d18);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// spinors: AoS half spinor (12 complex per site) <-> internal, nrhs fields.
// RHS r of the AoS data starts at aos + r*aos_stride (in complex numbers).
// ---------------------------------------------------------------------------
// `count` AoS spinors go to (or come from) RHS columns r0 .. r0+count-1 of the
// internal field (whose own RHS count is in the view). Threads run over RHS
// first (threadIdx.x) and sites second, as in the solver kernels, so the
// internal side of a warp is a contiguous run of 16-byte chunks.
template <int P>
__global__ void spinor_in_kernel(Geom g, int count, const double2* __restrict__ aos, size_t aos_stride, SpinorView dst,
                                 int r0) {
  typedef typename CompReal<P>::type R;
  const int r = blockIdx.y * blockDim.x + threadIdx.x;
  const int s = blockIdx.x * blockDim.y + threadIdx.y;
  if (s >= g.Vh || r >= count) return;
  const double2* p = aos + r * aos_stride + (size_t)s * 12;
  Spinor<R> v;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    double2 w = p[k];
    v.c[k] = mk((R)w.x, (R)w.y);
  }
  SpinorIO<P>::store(dst, s, r0 + r, v);
}

template <int P>
__global__ void spinor_out_kernel(Geom g, int count, CSpinorView src, double2* __restrict__ aos, size_t aos_stride,
                                  int r0) {
  typedef typename CompReal<P>::type R;
  const int r = blockIdx.y * blockDim.x + threadIdx.x;
  const int s = blockIdx.x * blockDim.y + threadIdx.y;
  if (s >= g.Vh || r >= count) return;
  Spinor<R> v;
  SpinorIO<P>::load(v, src, s, r0 + r);
  double2* p = aos + r * aos_stride + (size_t)s * 12;
#pragma unroll
  for (int k = 0; k < 12; k++) p[k] = make_double2((double)v.c[k].re, (double)v.c[k].im);
}

// 128 threads: up to 16 RHS lanes (the smallest power of two >= count) x sites
static void layout_shape(const Geom& g, int count, dim3* grid, dim3* block) {
  int rb = 1;
  while (rb < count && rb < 16) rb *= 2;
  *block = dim3(rb, 128 / rb);
  *grid = dim3(grid_x(g.Vh, 128 / rb), (count + rb - 1) / rb);
}

cudaError_t launch_spinor_in(int prec, const Geom& g, int count, const void* aos, size_t aos_stride, SpinorView dst,
                             cudaStream_t st, int r0) {
  dim3 block, grid;
  layout_shape(g, count, &grid, &block);
  const double2* a = static_cast<const double2*>(aos);
  switch (prec) {
    case PREC_DOUBLE: spinor_in_kernel<PREC_DOUBLE><<<grid, block, 0, st>>>(g, count, a, aos_stride, dst, r0); break;
    case PREC_SINGLE: spinor_in_kernel<PREC_SINGLE><<<grid, block, 0, st>>>(g, count, a, aos_stride, dst, r0); break;
    case PREC_HALF: spinor_in_kernel<PREC_HALF><<<grid, block, 0, st>>>(g, count, a, aos_stride, dst, r0); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_spinor_out(int prec, const Geom& g, int count, CSpinorView src, void* aos, size_t aos_stride,
                              cudaStream_t st, int r0) {
  dim3 block, grid;
  layout_shape(g, count, &grid, &block);
  double2* a = static_cast<double2*>(aos);
  switch (prec) {
    case PREC_DOUBLE: spinor_out_kernel<PREC_DOUBLE><<<grid, block, 0, st>>>(g, count, src, a, aos_stride, r0); break;
    case PREC_SINGLE: spinor_out_kernel<PREC_SINGLE><<<grid, block, 0, st>>>(g, count, src, a, aos_stride, r0); break;
    case PREC_HALF: spinor_out_kernel<PREC_HALF><<<grid, block, 0, st>>>(g, count, src, a, aos_stride, r0); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Loads the code of the FP64 spinor conversion kernels on the current device
// (with lazy module loading a kernel's module is otherwise loaded, and its
// device memory taken, at its first launch).
cudaError_t preload_spinor_io_f64() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, spinor_in_kernel<PREC_DOUBLE>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, spinor_out_kernel<PREC_DOUBLE>);
  return e;
}

// ---------------------------------------------------------------------------
// seeded synthetic fields (same streams and arithmetic as the CPU oracle)
// ---------------------------------------------------------------------------
QCU_D double unif01(uint64_t& s) { return (double)(sm64_next(s) >> 11) * 0x1.0p-53; }
QCU_D void gauss2(uint64_t& s, double& a, double& b) {
  double u1 = 1.0 - unif01(s);
  double u2 = unif01(s);
  double r = sqrt(-2.0 * log(u1));
  double th = 6.283185307179586476925286766559 * u2;
  a = r * cos(th);
  b = r * sin(th);
}

typedef Cplx<double> C64;

QCU_D void mm3(C64* r, const C64* a, const C64* b) {
  C64 t[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      C64 acc = mk(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; k++) acc += a[i * 3 + k] * b[k * 3 + j];
      t[i * 3 + j] = acc;
    }
#pragma unroll
  for (int i = 0; i < 9; i++) r[i] = t[i];
}

// U = exp(i*eps*H), H traceless Hermitian with Gaussian entries (diagonal:
// three N(0,1) minus their mean; off-diagonal: N(0,1) + i N(0,1)); scaling and
// squaring of a degree-12 Taylor series; Gram-Schmidt on rows 1-2 and
// row 3 = conj(row1 x row2), so det U = 1.
QCU_D void su3_from_stream(C64 u[9], uint64_t& st, double eps) {
  double gg[10];
#pragma unroll
  for (int k = 0; k < 5; k++) gauss2(st, gg[2 * k], gg[2 * k + 1]);
  C64 H[9];
  double mean = (gg[0] + gg[1] + gg[2]) / 3.0;
  H[0] = mk(gg[0] - mean, 0.0);
  H[4] = mk(gg[1] - mean, 0.0);
  H[8] = mk(gg[2] - mean, 0.0);
  H[1] = mk(gg[3], gg[4]); H[3] = conj(H[1]);
  H[2] = mk(gg[5], gg[6]); H[6] = conj(H[2]);
  H[5] = mk(gg[7], gg[8]); H[7] = conj(H[5]);
  C64 X[9];
  double nrm = 0;
  for (int i = 0; i < 9; i++) {
    X[i] = mk(-eps * H[i].im, eps * H[i].re);  // i*eps*H
    nrm += X[i].re * X[i].re + X[i].im * X[i].im;
  }
  nrm = sqrt(nrm);
  int k = 0;
  while (nrm > 0.25 && k < 30) { nrm *= 0.5; k++; }
  double sc = ldexp(1.0, -k);
  for (int i = 0; i < 9; i++) X[i] = sc * X[i];
  C64 E[9];
  for (int i = 0; i < 9; i++) E[i] = mk((i % 4 == 0) ? 1.0 : 0.0, 0.0);
  for (int n = 12; n >= 1; n--) {
    C64 T[9];
    mm3(T, X, E);
    for (int i = 0; i < 9; i++) E[i] = mk(((i % 4 == 0) ? 1.0 : 0.0) + T[i].re / (double)n, T[i].im / (double)n);
  }
  for (int s = 0; s < k; s++) mm3(E, E, E);
  double n0 = 0;
  for (int j = 0; j < 3; j++) n0 += E[j].re * E[j].re + E[j].im * E[j].im;
  n0 = 1.0 / sqrt(n0);
  for (int j = 0; j < 3; j++) u[j] = n0 * E[j];
  C64 ip = mk(0.0, 0.0);
  for (int j = 0; j < 3; j++) cmac_conj(ip, u[j], E[3 + j]);
  C64 r1[3];
  for (int j = 0; j < 3; j++) r1[j] = E[3 + j] - ip * u[j];
  double n1 = 0;
  for (int j = 0; j < 3; j++) n1 += r1[j].re * r1[j].re + r1[j].im * r1[j].im;
  n1 = 1.0 / sqrt(n1);
  for (int j = 0; j < 3; j++) u[3 + j] = n1 * r1[j];
  u[6] = conj(u[1] * u[5] - u[2] * u[4]);
  u[7] = conj(u[2] * u[3] - u[0] * u[5]);
  u[8] = conj(u[0] * u[4] - u[1] * u[3]);
}

__global__ void gauge_random_kernel(size_t nlinks, uint64_t seed, double eps, double2* out) {
  size_t l = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  uint64_t st = stream_init(seed, l);
  C64 u[9];
  su3_from_stream(u, st, eps);
  for (int i = 0; i < 9; i++) out[l * 9 + i] = make_double2(u[i].re, u[i].im);
}

__global__ void spinor_random_kernel(size_t nsites, uint64_t seed, double2* out) {
  size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsites) return;
  uint64_t st = stream_init(seed ^ 0xA0761D6478BD642Full, s);
  for (int k = 0; k < 12; k++) {
    double a, b;
    gauss2(st, a, b);
    out[s * 12 + k] = make_double2(a, b);
  }
}

// The links of slices t_first .. t_first + nslices - 1 (modulo the global
// time extent) of the global lattice's seeded field: link l of this slab has
// the stream of the global link with the same direction, parity and spatial
// site, so the union of the slabs is the field launch_gauge_random makes for
// the whole lattice.
__global__ void gauge_random_slab_kernel(size_t nlinks, size_t vh, size_t face, size_t vh_glob, int lt_glob,
                                         int t_first, uint64_t seed, double eps, double2* out) {
  size_t l = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nlinks) return;
  const size_t mp = l / vh, s = l - mp * vh;
  const size_t ts = s / face, rest = s - ts * face;
  const int tg = (int)(((long long)t_first + (long long)ts) % lt_glob + lt_glob) % lt_glob;
  uint64_t st = stream_init(seed, mp * vh_glob + (size_t)tg * face + rest);
  C64 u[9];
  su3_from_stream(u, st, eps);
  for (int i = 0; i < 9; i++) out[l * 9 + i] = make_double2(u[i].re, u[i].im);
}

cudaError_t launch_gauge_random_slab(const Geom& g, int lt_glob, int t_first, uint64_t seed, double eps, void* aos,
                                     cudaStream_t st) {
  const size_t n = (size_t)8 * g.Vh, face = (size_t)g.st;
  gauge_random_slab_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, g.Vh, face, face * lt_glob, lt_glob,
                                                                          t_first, seed, eps, static_cast<double2*>(aos));
  return cudaGetLastError();
}

// One full spinor of a slab (both parities, vh sites each) with the streams
// of the global field's sites: site s of parity p is global site
// p * vh_glob + offset + s.
__global__ void spinor_random_slab_kernel(size_t vh, size_t vh_glob, size_t offset, uint64_t seed, double2* out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * vh) return;
  const size_t p = i / vh, s = i - p * vh;
  uint64_t st = stream_init(seed ^ 0xA0761D6478BD642Full, p * vh_glob + offset + s);
  for (int k = 0; k < 12; k++) {
    double a, b;
    gauss2(st, a, b);
    out[i * 12 + k] = make_double2(a, b);
  }
}

cudaError_t launch_spinor_random_slab(const Geom& g, int lt_glob, int t0, uint64_t seed, void* aos, cudaStream_t st) {
  const size_t n = (size_t)2 * g.Vh, face = (size_t)g.st;
  spinor_random_slab_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g.Vh, face * lt_glob, face * t0, seed,
                                                                           static_cast<double2*>(aos));
  return cudaGetLastError();
}

cudaError_t launch_gauge_random(const Geom& g, uint64_t seed, double eps, void* aos, cudaStream_t st) {
  size_t n = (size_t)8 * g.Vh;
  gauge_random_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, seed, eps, static_cast<double2*>(aos));
  return cudaGetLastError();
}

cudaError_t launch_spinor_random(size_t nsites, uint64_t seed, void* aos, cudaStream_t st) {
  spinor_random_kernel<<<(unsigned)((nsites + 127) / 128), 128, 0, st>>>(nsites, seed, static_cast<double2*>(aos));
  return cudaGetLastError();
}

}  // namespace qcu
