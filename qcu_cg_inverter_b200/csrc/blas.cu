// Fused CG vector kernels. Each pass reads and writes every operand once and
// folds the dot products the solver needs into the same pass (single-pass
// deterministic reductions, qcu_reduce.cuh). The reference runs each BLAS
// call as its own kernel, with the complex scalar in device memory, a
// cudaDeviceSynchronize after every launch and a two-kernel tree reduction
// for every dot product (src/qcu_complex_computation.cu:10-133).
//
// Fields are one-parity (or, for full spinors, two consecutive parity blocks
// of Vh_pad sites); padding sites hold zeros and stay zero under every
// operation here.
#include "qcu_cg_state.cuh"
#include "qcu_fields.cuh"
#include "qcu_kernels.cuh"

namespace qcu {

#define QCU_SITE_RHS                                         \
  const int r = blockIdx.y * blockDim.x + threadIdx.x;       \
  const int s = blockIdx.x * blockDim.y + threadIdx.y;       \
  const bool valid = (s < nsites) && (r < nrhs) && (active == nullptr || active[r]);

template <class R> QCU_D double norm2(const Spinor<R>& v) {
  double n = 0.0;
#pragma unroll
  for (int k = 0; k < 12; k++) n += (double)v.c[k].re * v.c[k].re + (double)v.c[k].im * v.c[k].im;
  return n;
}

// p = r + beta p
template <int PA, int PS>
__global__ void __launch_bounds__(256) cg_p_kernel(int nsites, int nrhs, SpinorView p, CSpinorView rv,
                                                   const double* beta, const int* active) {
  typedef typename CompReal<PA>::type RA;
  typedef typename CompReal<PS>::type RS;
  QCU_SITE_RHS
  if (!valid) return;
  const RS b = (RS)beta[r];
  Spinor<RA> rr;
  Spinor<RS> pv;
  SpinorIO<PA>::load(rr, rv, s, r);
  SpinorIO<PS>::load(pv, p, s, r);
#pragma unroll
  for (int k = 0; k < 12; k++) {
    pv.c[k].re = (RS)rr.c[k].re + b * pv.c[k].re;
    pv.c[k].im = (RS)rr.c[k].im + b * pv.c[k].im;
  }
  SpinorIO<PS>::store(p, s, r, pv);
}

// dst = src (precision conversion); optional |dst|^2 (FinNone)
template <int PD, int PSRC, bool NORM>
__global__ void __launch_bounds__(256) convert_kernel(int nsites, int nrhs, SpinorView dst, CSpinorView src,
                                                      const int* active, ReduceArgs red) {
  typedef typename CompReal<PD>::type RD;
  typedef typename CompReal<PSRC>::type RS;
  QCU_SITE_RHS
  double nrm = 0.0;
  if (valid) {
    Spinor<RS> v;
    SpinorIO<PSRC>::load(v, src, s, r);
    Spinor<RD> w;
#pragma unroll
    for (int k = 0; k < 12; k++) w.c[k] = mk((RD)v.c[k].re, (RD)v.c[k].im);
    SpinorIO<PD>::store(dst, s, r, w);
    if (NORM) nrm = norm2(w);
  }
  if (NORM) {
    double v1[1] = {nrm};
    block_reduce_finish<1, FinNone>(v1, nrhs, red);
  }
}

// xhi += xlo ; xlo = 0
template <int PL>
__global__ void __launch_bounds__(256) accumulate_kernel(int nsites, int nrhs, SpinorView xhi, SpinorView xlo,
                                                         const int* active) {
  typedef typename CompReal<PL>::type RL;
  QCU_SITE_RHS
  if (!valid) return;
  Spinor<double> h;
  Spinor<RL> l;
  SpinorIO<PREC_DOUBLE>::load(h, xhi, s, r);
  SpinorIO<PL>::load(l, xlo, s, r);
#pragma unroll
  for (int k = 0; k < 12; k++) {
    h.c[k].re += (double)l.c[k].re;
    h.c[k].im += (double)l.c[k].im;
    l.c[k] = mk(RL(0), RL(0));
  }
  SpinorIO<PREC_DOUBLE>::store(xhi, s, r, h);
  SpinorIO<PL>::store(xlo, s, r, l);
}

// xhi += xlo ; xlo = 0 ; d = b - xhi (the start of r = bhat - Mhat xhi, which
// the next stencil completes as d + kappa^2 A^-1 D t)
template <int PL>
__global__ void __launch_bounds__(256) accumulate_res_kernel(int nsites, int nrhs, SpinorView xhi, SpinorView xlo,
                                                             CSpinorView b, SpinorView d, const int* active) {
  typedef typename CompReal<PL>::type RL;
  QCU_SITE_RHS
  if (!valid) return;
  Spinor<double> h, bv;
  Spinor<RL> l;
  SpinorIO<PREC_DOUBLE>::load(h, xhi, s, r);
  SpinorIO<PL>::load(l, xlo, s, r);
  SpinorIO<PREC_DOUBLE>::load(bv, b, s, r);
#pragma unroll
  for (int k = 0; k < 12; k++) {
    h.c[k].re += (double)l.c[k].re;
    h.c[k].im += (double)l.c[k].im;
    l.c[k] = mk(RL(0), RL(0));
    bv.c[k] = bv.c[k] - h.c[k];
  }
  SpinorIO<PREC_DOUBLE>::store(xhi, s, r, h);
  SpinorIO<PL>::store(xlo, s, r, l);
  SpinorIO<PREC_DOUBLE>::store(d, s, r, bv);
}

// f = 0 on the RHS in the mask (16-bit fields: norm 0 too)
template <int P>
__global__ void __launch_bounds__(256) zero_kernel(int nsites, int nrhs, SpinorView f, const int* active) {
  typedef typename CompReal<P>::type R;
  QCU_SITE_RHS
  if (!valid) return;
  Spinor<R> z;
#pragma unroll
  for (int k = 0; k < 12; k++) z.c[k] = mk(R(0), R(0));
  SpinorIO<P>::store(f, s, r, z);
}

// r = b - z (double), |r|^2 (FinNone)
__global__ void __launch_bounds__(256) residual_kernel(int nsites, int nrhs, SpinorView rv, CSpinorView b, CSpinorView z,
                                                       const int* active, ReduceArgs red) {
  QCU_SITE_RHS
  double nrm = 0.0;
  if (valid) {
    Spinor<double> bv, zv;
    SpinorIO<PREC_DOUBLE>::load(bv, b, s, r);
    SpinorIO<PREC_DOUBLE>::load(zv, z, s, r);
#pragma unroll
    for (int k = 0; k < 12; k++) bv.c[k] = bv.c[k] - zv.c[k];
    SpinorIO<PREC_DOUBLE>::store(rv, s, r, bv);
    nrm = norm2(bv);
  }
  double v[1] = {nrm};
  block_reduce_finish<1, FinNone>(v, nrhs, red);
}

// complex dot <x,y> = sum conj(x) y, two reals per RHS (FinNone)
template <int P>
__global__ void __launch_bounds__(256) cdot_kernel(int nsites, int nrhs, CSpinorView x, CSpinorView y, const int* active,
                                                   ReduceArgs red) {
  typedef typename CompReal<P>::type R;
  QCU_SITE_RHS
  double v[2] = {0.0, 0.0};
  if (valid) {
    Spinor<R> a, b;
    SpinorIO<P>::load(a, x, s, r);
    SpinorIO<P>::load(b, y, s, r);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      v[0] += (double)a.c[k].re * b.c[k].re + (double)a.c[k].im * b.c[k].im;
      v[1] += (double)a.c[k].re * b.c[k].im - (double)a.c[k].im * b.c[k].re;
    }
  }
  block_reduce_finish<2, FinNone>(v, nrhs, red);
}

// Complex updates of the reference CG flow (src/cg_inverter.cu:181-256), one
// RHS, double: x += a p ; r2 = r - a Ap ; <r2,r2>
__global__ void __launch_bounds__(256) ref_xr_kernel(int nsites, SpinorView x, CSpinorView p, CSpinorView rin,
                                                     CSpinorView ap, SpinorView r2, double2 a, ReduceArgs red) {
  const int nrhs = 1;
  const int* active = nullptr;
  QCU_SITE_RHS
  double v[2] = {0.0, 0.0};
  if (valid) {
    Spinor<double> xv, pv, rv, av;
    SpinorIO<PREC_DOUBLE>::load(xv, x, s, r);
    SpinorIO<PREC_DOUBLE>::load(pv, p, s, r);
    SpinorIO<PREC_DOUBLE>::load(rv, rin, s, 0);
    SpinorIO<PREC_DOUBLE>::load(av, ap, s, 0);
    const Cplx<double> A = mk(a.x, a.y);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      xv.c[k] += pv.c[k] * A;
      rv.c[k] -= av.c[k] * A;
      v[0] += rv.c[k].re * rv.c[k].re + rv.c[k].im * rv.c[k].im;
    }
    SpinorIO<PREC_DOUBLE>::store(x, s, r, xv);
    SpinorIO<PREC_DOUBLE>::store(r2, s, r, rv);
  }
  block_reduce_finish<2, FinNone>(v, nrhs, red);
}

// p = b p + r2 (complex b)
__global__ void __launch_bounds__(256) ref_p_kernel(int nsites, SpinorView p, CSpinorView r2, double2 b) {
  const int nrhs = 1;
  const int* active = nullptr;
  QCU_SITE_RHS
  if (!valid) return;
  Spinor<double> pv, rv;
  SpinorIO<PREC_DOUBLE>::load(pv, p, s, r);
  SpinorIO<PREC_DOUBLE>::load(rv, r2, s, r);
  const Cplx<double> B = mk(b.x, b.y);
#pragma unroll
  for (int k = 0; k < 12; k++) pv.c[k] = B * pv.c[k] + rv.c[k];
  SpinorIO<PREC_DOUBLE>::store(p, s, r, pv);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline dim3 blk(LaunchShape sh) { return dim3(sh.Rb, sh.Sb); }
static inline dim3 grd(int nsites, int nrhs, LaunchShape sh) {
  return dim3(grid_x(nsites, sh.Sb), (nrhs + sh.Rb - 1) / sh.Rb);
}

cudaError_t launch_cg_p(int pa, int ps, int nsites, int nrhs, SpinorView p, CSpinorView r, const double* beta,
                        const int* active, LaunchShape sh, cudaStream_t st) {
  dim3 b = blk(sh), g = grd(nsites, nrhs, sh);
#define QCU_P(A, S) cg_p_kernel<A, S><<<g, b, 0, st>>>(nsites, nrhs, p, r, beta, active)
  if (pa == PREC_DOUBLE && ps == PREC_DOUBLE) QCU_P(PREC_DOUBLE, PREC_DOUBLE);
  else if (pa == PREC_SINGLE && ps == PREC_SINGLE) QCU_P(PREC_SINGLE, PREC_SINGLE);
  else if (pa == PREC_SINGLE && ps == PREC_HALF) QCU_P(PREC_SINGLE, PREC_HALF);
  else if (pa == PREC_HALF && ps == PREC_HALF) QCU_P(PREC_HALF, PREC_HALF);
  else return cudaErrorInvalidValue;
#undef QCU_P
  return cudaGetLastError();
}

cudaError_t launch_convert(int pd, int psrc, int nsites, int nrhs, SpinorView dst, CSpinorView src, const int* active,
                           const ReduceArgs* red, LaunchShape sh, cudaStream_t st) {
  dim3 b = blk(sh), g = grd(nsites, nrhs, sh);
  ReduceArgs rd = red ? *red : ReduceArgs{nullptr, nullptr, nullptr, nullptr};
#define QCU_CV(D, S)                                                                                   \
  if (red) convert_kernel<D, S, true><<<g, b, 0, st>>>(nsites, nrhs, dst, src, active, rd);            \
  else convert_kernel<D, S, false><<<g, b, 0, st>>>(nsites, nrhs, dst, src, active, rd);
  if (pd == PREC_DOUBLE && psrc == PREC_DOUBLE) { QCU_CV(PREC_DOUBLE, PREC_DOUBLE) }
  else if (pd == PREC_SINGLE && psrc == PREC_DOUBLE) { QCU_CV(PREC_SINGLE, PREC_DOUBLE) }
  else if (pd == PREC_HALF && psrc == PREC_DOUBLE) { QCU_CV(PREC_HALF, PREC_DOUBLE) }
  else if (pd == PREC_HALF && psrc == PREC_SINGLE) { QCU_CV(PREC_HALF, PREC_SINGLE) }
  else if (pd == PREC_SINGLE && psrc == PREC_SINGLE) { QCU_CV(PREC_SINGLE, PREC_SINGLE) }
  else if (pd == PREC_DOUBLE && psrc == PREC_SINGLE) { QCU_CV(PREC_DOUBLE, PREC_SINGLE) }
  else if (pd == PREC_DOUBLE && psrc == PREC_HALF) { QCU_CV(PREC_DOUBLE, PREC_HALF) }
  else if (pd == PREC_HALF && psrc == PREC_HALF) { QCU_CV(PREC_HALF, PREC_HALF) }
  else if (pd == PREC_SINGLE && psrc == PREC_HALF) { QCU_CV(PREC_SINGLE, PREC_HALF) }
  else return cudaErrorInvalidValue;
#undef QCU_CV
  return cudaGetLastError();
}

cudaError_t launch_accumulate(int pl, int nsites, int nrhs, SpinorView xhi, SpinorView xlo, const int* active,
                              LaunchShape sh, cudaStream_t st) {
  dim3 b = blk(sh), g = grd(nsites, nrhs, sh);
  if (pl == PREC_DOUBLE) accumulate_kernel<PREC_DOUBLE><<<g, b, 0, st>>>(nsites, nrhs, xhi, xlo, active);
  else if (pl == PREC_SINGLE) accumulate_kernel<PREC_SINGLE><<<g, b, 0, st>>>(nsites, nrhs, xhi, xlo, active);
  else if (pl == PREC_HALF) accumulate_kernel<PREC_HALF><<<g, b, 0, st>>>(nsites, nrhs, xhi, xlo, active);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_zero(int prec, int nsites, int nrhs, SpinorView f, const int* active, LaunchShape sh,
                        cudaStream_t st) {
  dim3 b = blk(sh), g = grd(nsites, nrhs, sh);
  switch (prec) {
    case PREC_DOUBLE: zero_kernel<PREC_DOUBLE><<<g, b, 0, st>>>(nsites, nrhs, f, active); break;
    case PREC_SINGLE: zero_kernel<PREC_SINGLE><<<g, b, 0, st>>>(nsites, nrhs, f, active); break;
    case PREC_HALF: zero_kernel<PREC_HALF><<<g, b, 0, st>>>(nsites, nrhs, f, active); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_accumulate_res(int pl, int nsites, int nrhs, SpinorView xhi, SpinorView xlo, CSpinorView b,
                                  SpinorView d, const int* active, LaunchShape sh, cudaStream_t st) {
  dim3 bl = blk(sh), g = grd(nsites, nrhs, sh);
  if (pl == PREC_DOUBLE) accumulate_res_kernel<PREC_DOUBLE><<<g, bl, 0, st>>>(nsites, nrhs, xhi, xlo, b, d, active);
  else if (pl == PREC_SINGLE) accumulate_res_kernel<PREC_SINGLE><<<g, bl, 0, st>>>(nsites, nrhs, xhi, xlo, b, d, active);
  else if (pl == PREC_HALF) accumulate_res_kernel<PREC_HALF><<<g, bl, 0, st>>>(nsites, nrhs, xhi, xlo, b, d, active);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_residual(int nsites, int nrhs, SpinorView r, CSpinorView b, CSpinorView z, const int* active,
                            const ReduceArgs& red, LaunchShape sh, cudaStream_t st) {
  residual_kernel<<<grd(nsites, nrhs, sh), blk(sh), 0, st>>>(nsites, nrhs, r, b, z, active, red);
  return cudaGetLastError();
}

cudaError_t launch_cdot(int prec, int nsites, int nrhs, CSpinorView x, CSpinorView y, const int* active,
                        const ReduceArgs& red, LaunchShape sh, cudaStream_t st) {
  dim3 b = blk(sh), g = grd(nsites, nrhs, sh);
  switch (prec) {
    case PREC_DOUBLE: cdot_kernel<PREC_DOUBLE><<<g, b, 0, st>>>(nsites, nrhs, x, y, active, red); break;
    case PREC_SINGLE: cdot_kernel<PREC_SINGLE><<<g, b, 0, st>>>(nsites, nrhs, x, y, active, red); break;
    case PREC_HALF: cdot_kernel<PREC_HALF><<<g, b, 0, st>>>(nsites, nrhs, x, y, active, red); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_ref_xr(int nsites, SpinorView x, CSpinorView p, CSpinorView r, CSpinorView ap, SpinorView r2,
                          double2 a, const ReduceArgs& red, LaunchShape sh, cudaStream_t st) {
  ref_xr_kernel<<<grd(nsites, 1, sh), blk(sh), 0, st>>>(nsites, x, p, r, ap, r2, a, red);
  return cudaGetLastError();
}

cudaError_t launch_ref_p(int nsites, SpinorView p, CSpinorView r2, double2 b, LaunchShape sh, cudaStream_t st) {
  ref_p_kernel<<<grd(nsites, 1, sh), blk(sh), 0, st>>>(nsites, p, r2, b);
  return cudaGetLastError();
}

}  // namespace qcu
