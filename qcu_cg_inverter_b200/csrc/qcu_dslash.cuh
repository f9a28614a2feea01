// The Wilson hopping term on one checkerboard, as a device function shared by
// all stencil kernels.
//
//   out(x) = sum_mu (1 - f g_mu) U_mu(x) in(x+mu) + (1 + f g_mu) U_mu(x-mu)^dag in(x-mu)
//
// f = +1 (D) or -1 (D^dag, which is exactly the adjoint of D), DeGrand-Rossi
// gamma matrices. Each direction is a two-component spin projection, two SU(3)
// mat-vecs and the spin reconstruction, with the same projector rows as the
// reference hopping kernel (src/qcu_clover_dslash.cu:599-768, flag = f). The
// reference has no kappa and no overall sign; neither has this function.
// bc_t multiplies every hop that crosses the t boundary (-1: antiperiodic).
#pragma once
#include "qcu_fields.cuh"

namespace qcu {

template <class R> struct Half2 {
  Cplx<R> h0[3], h1[3];
};

// h = P_mu^{fwd/bwd} psi. FWD: (1 - F g_mu), BWD: (1 + F g_mu).
template <int MU, bool FWD, int F, class R>
QCU_D void project(Half2<R>& h, const Spinor<R>& p) {
  // sign of the projector term: S = -F forward, +F backward
  constexpr int S = FWD ? -F : F;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const Cplx<R> p0 = p.c[c], p1 = p.c[3 + c], p2 = p.c[6 + c], p3 = p.c[9 + c];
    if constexpr (MU == 0) {  // h0 = p0 + S i p3, h1 = p1 + S i p2
      h.h0[c] = S > 0 ? p0 + mul_i(p3) : p0 - mul_i(p3);
      h.h1[c] = S > 0 ? p1 + mul_i(p2) : p1 - mul_i(p2);
    } else if constexpr (MU == 1) {  // h0 = p0 - S p3, h1 = p1 + S p2
      h.h0[c] = S > 0 ? p0 - p3 : p0 + p3;
      h.h1[c] = S > 0 ? p1 + p2 : p1 - p2;
    } else if constexpr (MU == 2) {  // h0 = p0 + S i p2, h1 = p1 - S i p3
      h.h0[c] = S > 0 ? p0 + mul_i(p2) : p0 - mul_i(p2);
      h.h1[c] = S > 0 ? p1 - mul_i(p3) : p1 + mul_i(p3);
    } else {  // h0 = p0 + S p2, h1 = p1 + S p3
      h.h0[c] = S > 0 ? p0 + p2 : p0 - p2;
      h.h1[c] = S > 0 ? p1 + p3 : p1 - p3;
    }
  }
}

// out += reconstruct(a = U h0, b = U h1)
template <int MU, bool FWD, int F, class R>
QCU_D void reconstruct(Spinor<R>& o, const Cplx<R> a[3], const Cplx<R> b[3]) {
  constexpr int S = FWD ? -F : F;  // same sign convention as project()
#pragma unroll
  for (int c = 0; c < 3; c++) {
    o.c[c] += a[c];
    o.c[3 + c] += b[c];
    if constexpr (MU == 0) {  // o2 -= S i b, o3 -= S i a
      if (S > 0) { o.c[6 + c] -= mul_i(b[c]); o.c[9 + c] -= mul_i(a[c]); }
      else { o.c[6 + c] += mul_i(b[c]); o.c[9 + c] += mul_i(a[c]); }
    } else if constexpr (MU == 1) {  // o2 += S b, o3 -= S a
      if (S > 0) { o.c[6 + c] += b[c]; o.c[9 + c] -= a[c]; }
      else { o.c[6 + c] -= b[c]; o.c[9 + c] += a[c]; }
    } else if constexpr (MU == 2) {  // o2 -= S i a, o3 += S i b
      if (S > 0) { o.c[6 + c] -= mul_i(a[c]); o.c[9 + c] += mul_i(b[c]); }
      else { o.c[6 + c] += mul_i(a[c]); o.c[9 + c] -= mul_i(b[c]); }
    } else {  // o2 += S a, o3 += S b
      if (S > 0) { o.c[6 + c] += a[c]; o.c[9 + c] += b[c]; }
      else { o.c[6 + c] -= a[c]; o.c[9 + c] -= b[c]; }
    }
  }
}

template <class R>
QCU_D void su3_mul(Cplx<R> o[3], const Link<R>& U, const Cplx<R> v[3]) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    Cplx<R> acc = U.u[i * 3] * v[0];
    cmac(acc, U.u[i * 3 + 1], v[1]);
    cmac(acc, U.u[i * 3 + 2], v[2]);
    o[i] = acc;
  }
}
template <class R>
QCU_D void su3_dag_mul(Cplx<R> o[3], const Link<R>& U, const Cplx<R> v[3]) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    Cplx<R> acc = mk(R(0), R(0));
    cmac_conj(acc, U.u[i], v[0]);
    cmac_conj(acc, U.u[3 + i], v[1]);
    cmac_conj(acc, U.u[6 + i], v[2]);
    o[i] = acc;
  }
}

template <class R> QCU_D void scale_half(Half2<R>& h, R s) {
#pragma unroll
  for (int c = 0; c < 3; c++) { h.h0[c] = s * h.h0[c]; h.h1[c] = s * h.h1[c]; }
}

// Loads the neighbour spinor and projects it, times `phase` (the time
// boundary factor, or 1). For 16-bit storage the per-site norm is applied to
// the six projected components instead of the twelve stored ones.
template <int PS, int MU, bool FWD, int F, class R>
QCU_D void load_project(Half2<R>& h, const CSpinorView& in, int s, int r, R phase) {
  if constexpr (PS == PREC_HALF) {
    Spinor<float> raw;
    float nm = SpinorIO<PREC_HALF>::load_raw(raw, in, s, r) * (float)phase;
    Half2<float> hf;
    project<MU, FWD, F>(hf, raw);
    scale_half(hf, nm);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      h.h0[c] = mk((R)hf.h0[c].re, (R)hf.h0[c].im);
      h.h1[c] = mk((R)hf.h1[c].re, (R)hf.h1[c].im);
    }
  } else {
    Spinor<R> p;
    SpinorIO<PS>::load(p, in, s, r);
    project<MU, FWD, F>(h, p);
    if (MU == 3 && phase != R(1)) scale_half(h, phase);
  }
}

// One direction (both hops) of the stencil: PS = spinor precision, PL = link
// storage format.
template <int PS, int PL, int MU, int F, class R>
QCU_D void hop_dir(Spinor<R>& o, const Geom& g, const Nbrs& nb, int parity, int s, int r,
                   const CSpinorView& in, const void* gauge, R bc_t) {
  Link<R> U;
  Half2<R> h;
  Cplx<R> a[3], b[3];
  // forward: U_mu(x) in(x+mu)
  LinkIO<PL>::load(U, gauge, g.Vh_pad, MU, parity, s);
  load_project<PS, MU, true, F>(h, in, nb.fwd[MU], r, (MU == 3 && nb.t == g.Lt - 1) ? bc_t : R(1));
  su3_mul(a, U, h.h0);
  su3_mul(b, U, h.h1);
  reconstruct<MU, true, F>(o, a, b);
  // backward: U_mu(x-mu)^dag in(x-mu); the link lives on the other parity
  LinkIO<PL>::load(U, gauge, g.Vh_pad, MU, 1 - parity, nb.bwd[MU]);
  load_project<PS, MU, false, F>(h, in, nb.bwd[MU], r, (MU == 3 && nb.t == 0) ? bc_t : R(1));
  su3_dag_mul(a, U, h.h0);
  su3_dag_mul(b, U, h.h1);
  reconstruct<MU, false, F>(o, a, b);
}

template <int PS, int PL, bool DAG, class R>
QCU_D void hop(Spinor<R>& o, const Geom& g, int parity, int s, int r, const CSpinorView& in,
               const void* gauge, R bc_t) {
  constexpr int F = DAG ? -1 : 1;
#pragma unroll
  for (int k = 0; k < 12; k++) o.c[k] = mk(R(0), R(0));
  const Nbrs nb = neighbours(g, s, parity);
  hop_dir<PS, PL, 0, F>(o, g, nb, parity, s, r, in, gauge, bc_t);
  hop_dir<PS, PL, 1, F>(o, g, nb, parity, s, r, in, gauge, bc_t);
  hop_dir<PS, PL, 2, F>(o, g, nb, parity, s, r, in, gauge, bc_t);
  hop_dir<PS, PL, 3, F>(o, g, nb, parity, s, r, in, gauge, bc_t);
}

}  // namespace qcu
