// Fused Wilson-clover stencil kernels: hop + optional clover, xpay, second
// output and per-RHS norm reduction, for double, single and 16-bit storage.
//
// One thread per (site, right-hand side). Threads of a warp that share a site
// (rhs lanes, threadIdx.x) load the same link addresses, which the memory
// system serves once; adjacent rhs lanes read adjacent spinor chunks.
#pragma once
#include "qcu_cg_state.cuh"
#include "qcu_dslash.cuh"
#include "qcu_kernels.cuh"

namespace qcu {

typedef void (*DslashKernelFn)(const DslashArgs);

// Minimum resident blocks (of up to 256 threads) per SM requested from the
// register allocator: 2 caps the stencil at 128 registers. Measured on B200 at
// 32^3x64 against no cap and an 85-register cap: equal or faster for every
// precision and epilogue (16-bit fused: 203 vs 235 us; FP64 hop 232 vs 240
// us), while 85 registers spill (FP64 hop 509 us).
#ifndef QCU_DSLASH_MINB
#define QCU_DSLASH_MINB 2
#endif
// The 16-bit kernel with the second clover output (the CG's fused Mhat half
// step) gets an 85-register cap instead: measured at 32^4, 16 RHS: 1246 vs
// 1348 us (24 instead of 16 resident warps; 36 bytes of spills), while the
// other 16-bit kernels are faster at 128 registers (hop: 677 vs 742 us).
#ifndef QCU_DSLASH_MINB16_OUT2
#define QCU_DSLASH_MINB16_OUT2 3
#endif
// likewise the hop + A^-1 kernel (measured in the 48-RHS 24^3x48 solve:
// 0.600 vs 0.605 s); the kernel with the fused CG update stays at 128
// registers (0.660 s with the 85-register cap)
#ifndef QCU_DSLASH_MINB16_CPRE
#define QCU_DSLASH_MINB16_CPRE 3
#endif
#ifndef QCU_DSLASH_MINB16_CGXR
#define QCU_DSLASH_MINB16_CGXR 2
#endif
// whether the single-RHS 16-bit kernels take the same caps as the batched ones
// (measured: no; 16^3x32 solve 3.88 vs 3.63 ms, 32^4 fused stencil 121 vs 114 us)
#ifndef QCU_DSLASH_CAP_1RHS
#define QCU_DSLASH_CAP_1RHS 0
#endif
// FP64 stencils (the FP64 solver and every reliable update): no register cap
// beyond the 255 of the architecture, since the cap of 128 made them spill
// (measured: FP64 hop at 32^3x64 249 -> 216 us; FP64 16^3x32 solve 7.21 -> 6.91 ms)
#ifndef QCU_DSLASH_MINB64
#define QCU_DSLASH_MINB64 1
#endif
// RHS-paired kernels (two right-hand sides per thread): blocks of at most
// 128 threads (half of the 256-slot RHS x site tile); 3 blocks per SM allow
// 168 registers
#ifndef QCU_DSLASH_MINB_PAIR
#define QCU_DSLASH_MINB_PAIR 4
#endif
#ifndef QCU_DSLASH_MINB_PAIR_OUT2
#define QCU_DSLASH_MINB_PAIR_OUT2 QCU_DSLASH_MINB_PAIR
#endif
constexpr int dslash_maxt(int op) { return op_pair(op) ? 128 : 256; }
// the compact single-RHS family (OP_HALF_1): 128 registers. Measured at
// 32^3x64 against the 85-register cap (80 used, 28 B spilled): K2 170 vs 164
// us, K4 134 vs 136 us, the solve 29.1 vs 29.2 ms - even, so no cap
#ifndef QCU_DSLASH_MINB_C1
#define QCU_DSLASH_MINB_C1 QCU_DSLASH_MINB
#endif
// batched FP64 launches (reliable updates of multi-RHS solves): the
// 128-register cap with row-at-a-time reconstruction (measured in the 48-RHS
// 24^3x48 solve: 0.556 vs 0.568 s)
#ifndef QCU_DSLASH_MINB64_BATCH
#define QCU_DSLASH_MINB64_BATCH 2
#endif
constexpr int dslash_minb(int op, int epi) {
  return op == OP_HALF_1 ? QCU_DSLASH_MINB_C1
         : op == OP_DOUBLE ? QCU_DSLASH_MINB64
         : op == OP_DOUBLE_BATCH ? QCU_DSLASH_MINB64_BATCH
         : op_pair(op) ? ((epi & EPI_OUT2) ? QCU_DSLASH_MINB_PAIR_OUT2 : QCU_DSLASH_MINB_PAIR)
         : (op_spinor_prec(op) != PREC_HALF || ((op == OP_HALF_FAST_1 || op == OP_HALF_1) && !QCU_DSLASH_CAP_1RHS))
             ? QCU_DSLASH_MINB
         : (epi & EPI_OUT2)              ? QCU_DSLASH_MINB16_OUT2
         : (epi & EPI_CGXR)              ? QCU_DSLASH_MINB16_CGXR
         : (epi == EPI_CPRE)             ? QCU_DSLASH_MINB16_CPRE
                                         : QCU_DSLASH_MINB;
}

// |v|^2 of one site: in the spinor's own precision (FP32 sums of 24 terms for
// the sloppy operators, no per-term conversion to double), then FP64 across
// sites in the block reduction
template <class R> QCU_D double site_norm2(const Spinor<R>& v) {
  R n = R(0);
#pragma unroll
  for (int k = 0; k < 12; k++) {
    n = fma(v.c[k].re, v.c[k].re, n);
    n = fma(v.c[k].im, v.c[k].im, n);
  }
  return (double)n;
}

// Clover field of RHS r: its slot in the bank, or nullptr for a negative slot
// index (no clover term for that RHS, A = 1), so Wilson and clover systems can
// share a batch.
QCU_D const void* clover_of(const DslashArgs& a, int r) {
  if (!a.clover_idx) return a.clover;
  const int ci = a.clover_idx[r];
  return ci >= 0 ? static_cast<const char*>(a.clover) + a.clover_stride * (size_t)ci : nullptr;
}

}  // namespace qcu
#include "qcu_dslash_pair.cuh"
namespace qcu {

// v <- C v, block-paired, for the clover storage of link format PL's operator
// (FP32 block-interleaved with the 18-real links, 16-bit with the 16-bit links)
template <int PL>
QCU_D void clover_block(SpinBlock& v, const void* clov, int Vh_pad, int parity, int s) {
  if constexpr (PL == LINK_HALF_RAW)
    clover_apply_block16(v, clov, Vh_pad, parity, s);
  else
    clover_apply_block(v, clov, Vh_pad, parity, s);
}

// One output site and RHS of a single-RHS 16-bit operator: the hop and every
// epilogue in block-paired FP32 instructions. PL = LINK_SINGLE18: the fast
// storage (FP32 18-real links, FP32 block-interleaved clover); PL =
// LINK_HALF_RAW: the compact one (16-bit 12-real links, 16-bit clover). Same
// arithmetic per component as the generic body below; the norms are summed in
// FP32 before the FP64 block sums.
template <int PL, bool DAG, int EPI>
QCU_D void site_half_fast(const DslashArgs& a, int s, int r, double& nrm) {
  SpinBlock o;
  hop_half_block<PL, DAG>(o, a.g, a.parity, s, r, a.in, a.gauge, (float)a.bc_t);
  const void* clov = (EPI & (EPI_CPRE | EPI_CX | EPI_CPOST | EPI_OUT2)) ? clover_of(a, r) : nullptr;
  if (EPI & EPI_CPRE)
    if (clov) clover_block<PL>(o, clov, a.g.Vh_pad, a.parity, s);
  if (EPI & EPI_XPAY) {
    const float2 c = splat2(a.coef ? (float)a.coef[r] : (float)a.coef0);
    SpinBlock xv;
    load16_block(xv, a.x, s, r);
    if (EPI & EPI_CX)
      if (clov) clover_block<PL>(xv, clov, a.g.Vh_pad, a.parity, s);
#pragma unroll
    for (int j = 0; j < 6; j++) {
      o.re[j] = ffma2(c, o.re[j], xv.re[j]);
      o.im[j] = ffma2(c, o.im[j], xv.im[j]);
    }
    if (EPI & EPI_CPOST)
      if (clov) clover_block<PL>(o, clov, a.g.Vh_pad, a.parity, s);
  }
  if constexpr ((EPI & EPI_CGXR) != 0) {
    // x += alpha p, r -= alpha out (the out of this kernel is the CG's z)
    const float al = (float)a.alpha[r];
    Spinor<float> xv, rv, pv;
    SpinorIO<acc_prec(PREC_HALF)>::load(xv, a.xacc, s, r);
    SpinorIO<acc_prec(PREC_HALF)>::load(rv, a.racc, s, r);
    SpinorIO<PREC_HALF>::load(pv, a.pvec, s, r);
    float n = 0.f;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const Cplx<float> z = block_comp(o, k);
      xv.c[k].re += al * pv.c[k].re;
      xv.c[k].im += al * pv.c[k].im;
      rv.c[k].re -= al * z.re;
      rv.c[k].im -= al * z.im;
      n = fmaf(rv.c[k].re, rv.c[k].re, n);
      n = fmaf(rv.c[k].im, rv.c[k].im, n);
    }
    SpinorIO<acc_prec(PREC_HALF)>::store(a.xacc, s, r, xv);
    SpinorIO<acc_prec(PREC_HALF)>::store(a.racc, s, r, rv);
    nrm = n;
  } else {
    store16_block(a.out, s, r, o);
    if (EPI & EPI_NORM) nrm = norm2_block(o);
  }
  if (EPI & EPI_OUT2) {
    if (clov) clover_block<PL>(o, clov, a.g.Vh_pad, a.parity, s);
    store16_block(a.out2, s, r, o);
  }
}

// One (site, RHS) per thread.
template <int OP, bool DAG, int EPI, class Fin>
QCU_D void dslash_site_body(const DslashArgs& a) {
  constexpr int PS = op_spinor_prec(OP), PL = op_link_format(OP), PC = op_clover_prec(OP);
  typedef typename CompReal<PS>::type R;
  const TileCoord tc = stencil_tile(a);
  const int r = tc.rhs * blockDim.x + threadIdx.x;
  const int s = stencil_site0(a, tc) + threadIdx.y;
  const bool valid = (s < stencil_slim(a)) && (r < a.nrhs) && (a.active == nullptr || a.active[r]);
  double nrm = 0.0;
  // single-RHS launches of the fast 16-bit operator: block-paired epilogues
  // (measured: 16^3x32 solve 3.70 vs 3.88 ms); with many RHS per launch the
  // generic body at the 85-register cap is faster (48-RHS batch 0.592 vs 0.606 s)
  if (OP == OP_HALF_FAST_1 && valid) {
    site_half_fast<LINK_SINGLE18, DAG, EPI>(a, s, r, nrm);
  } else if (OP == OP_HALF_1 && valid) {
    site_half_fast<LINK_HALF_RAW, DAG, EPI>(a, s, r, nrm);
  } else if (valid) {
    Spinor<R> o;
    hop<PS, PL, DAG, OP == OP_DOUBLE_BATCH>(o, a.g, a.parity, s, r, a.in, a.gauge, (R)a.bc_t);
    const void* clov = (EPI & (EPI_CPRE | EPI_CX | EPI_CPOST | EPI_OUT2)) ? clover_of(a, r) : nullptr;
    if (EPI & EPI_CPRE)
      if (clov) clover_apply_site<PC>(o, clov, a.g.Vh_pad, a.parity, s);
    if (EPI & EPI_XPAY) {
      const R c = a.coef ? (R)a.coef[r] : (R)a.coef0;
      Spinor<R> xv;
      SpinorIO<PS>::load(xv, a.x, s, r);
      if (EPI & EPI_CX)
        if (clov) clover_apply_site<PC>(xv, clov, a.g.Vh_pad, a.parity, s);
#pragma unroll
      for (int k = 0; k < 12; k++) o.c[k] = xv.c[k] + c * o.c[k];
      if (EPI & EPI_CPOST)
        if (clov) clover_apply_site<PC>(o, clov, a.g.Vh_pad, a.parity, s);
    }
    if constexpr ((EPI & EPI_CGXR) != 0) {
      // x += alpha p, r -= alpha out (the out of this kernel is the CG's z)
      constexpr int PA = acc_prec(PS);
      typedef typename CompReal<PA>::type RA;
      const RA al = (RA)a.alpha[r];
      Spinor<RA> xv, rv;
      Spinor<R> pv;
      SpinorIO<PA>::load(xv, a.xacc, s, r);
      SpinorIO<PA>::load(rv, a.racc, s, r);
      SpinorIO<PS>::load(pv, a.pvec, s, r);
#pragma unroll
      for (int k = 0; k < 12; k++) {
        xv.c[k].re += al * (RA)pv.c[k].re;
        xv.c[k].im += al * (RA)pv.c[k].im;
        rv.c[k].re -= al * (RA)o.c[k].re;
        rv.c[k].im -= al * (RA)o.c[k].im;
      }
      SpinorIO<PA>::store(a.xacc, s, r, xv);
      SpinorIO<PA>::store(a.racc, s, r, rv);
      nrm = site_norm2(rv);
    } else {
      SpinorIO<PS>::store(a.out, s, r, o);
      if (EPI & EPI_NORM) nrm = site_norm2(o);
    }
    if (EPI & EPI_OUT2) {
      if (clov) clover_apply_site<PC>(o, clov, a.g.Vh_pad, a.parity, s);
      SpinorIO<PS>::store(a.out2, s, r, o);
    }
  }
  if (EPI & (EPI_NORM | EPI_CGXR)) {
    double v[1] = {nrm};
    block_reduce_finish<1, Fin>(v, a.nrhs, a.red, tc);
  }
}

// OP selects the storage of spinors, links and clover (OpVariant), and for the
// fast 16-bit storage the kernel family: OP_HALF_FAST_2(T, Z) serve two RHS per
// thread (qcu_dslash_pair.cuh), the others one.
template <int OP, bool DAG, int EPI, class Fin>
__global__ void __launch_bounds__(dslash_maxt(OP), dslash_minb(OP, EPI)) dslash_kernel(const DslashArgs a) {
  if constexpr (op_pair(OP))
    dslash_pair_body<op_staged(OP), DAG, EPI, Fin>(a);
  else
    dslash_site_body<OP, DAG, EPI, Fin>(a);
}

template <int P, bool DAG>
static DslashKernelFn pick(int epi, int fin) {
#define QCU_CASE(E)                                                                     \
  case (E):                                                                             \
    if constexpr (((E)&EPI_CGXR) != 0) {                                                \
      if (fin == FIN_CG_BETA) return dslash_kernel<P, DAG, (E), FinCgBeta>;             \
      return fin == FIN_NONE ? dslash_kernel<P, DAG, (E), FinNone> : nullptr;           \
    } else if constexpr (((E)&EPI_NORM) != 0) {                                         \
      if (fin == FIN_CG_ALPHA) return dslash_kernel<P, DAG, (E), FinCgAlpha>;           \
      return dslash_kernel<P, DAG, (E), FinNone>;                                       \
    } else {                                                                            \
      return dslash_kernel<P, DAG, (E), FinNone>;                                       \
    }
  switch (epi) {
    QCU_CASE(0)
    QCU_CASE(EPI_CPRE)
    QCU_CASE(EPI_XPAY)
    QCU_CASE(EPI_XPAY | EPI_CX)
    QCU_CASE(EPI_XPAY | EPI_CPOST)
    QCU_CASE(EPI_CPRE | EPI_XPAY)
    QCU_CASE(EPI_CPRE | EPI_XPAY | EPI_NORM)
    QCU_CASE(EPI_CPRE | EPI_XPAY | EPI_OUT2)
    QCU_CASE(EPI_CPRE | EPI_XPAY | EPI_OUT2 | EPI_NORM)
    QCU_CASE(EPI_XPAY | EPI_NORM)
    QCU_CASE(EPI_XPAY | EPI_CGXR)
    default:
      return nullptr;
  }
#undef QCU_CASE
}

}  // namespace qcu
