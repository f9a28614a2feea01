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

// out += reconstruct(a = U h0, b = U h1), colour row c
template <int MU, bool FWD, int F, class R>
QCU_D void reconstruct_row(Spinor<R>& o, int c, const Cplx<R>& a, const Cplx<R>& b) {
  constexpr int S = FWD ? -F : F;  // same sign convention as project()
  o.c[c] += a;
  o.c[3 + c] += b;
  if constexpr (MU == 0) {  // o2 -= S i b, o3 -= S i a
    if (S > 0) { o.c[6 + c] -= mul_i(b); o.c[9 + c] -= mul_i(a); }
    else { o.c[6 + c] += mul_i(b); o.c[9 + c] += mul_i(a); }
  } else if constexpr (MU == 1) {  // o2 += S b, o3 -= S a
    if (S > 0) { o.c[6 + c] += b; o.c[9 + c] -= a; }
    else { o.c[6 + c] -= b; o.c[9 + c] += a; }
  } else if constexpr (MU == 2) {  // o2 -= S i a, o3 += S i b
    if (S > 0) { o.c[6 + c] -= mul_i(a); o.c[9 + c] += mul_i(b); }
    else { o.c[6 + c] += mul_i(a); o.c[9 + c] -= mul_i(b); }
  } else {  // o2 += S a, o3 += S b
    if (S > 0) { o.c[6 + c] += a; o.c[9 + c] += b; }
    else { o.c[6 + c] -= a; o.c[9 + c] -= b; }
  }
}
template <int MU, bool FWD, int F, class R>
QCU_D void reconstruct(Spinor<R>& o, const Cplx<R> a[3], const Cplx<R> b[3]) {
#pragma unroll
  for (int c = 0; c < 3; c++) reconstruct_row<MU, FWD, F>(o, c, a[c], b[c]);
}

// row i of U v and of U^dag v
template <class R>
QCU_D Cplx<R> su3_row(const Link<R>& U, const Cplx<R> v[3], int i) {
  Cplx<R> acc = U.u[i * 3] * v[0];
  cmac(acc, U.u[i * 3 + 1], v[1]);
  cmac(acc, U.u[i * 3 + 2], v[2]);
  return acc;
}
template <class R>
QCU_D Cplx<R> su3_dag_row(const Link<R>& U, const Cplx<R> v[3], int i) {
  Cplx<R> acc = mk(R(0), R(0));
  cmac_conj(acc, U.u[i], v[0]);
  cmac_conj(acc, U.u[3 + i], v[1]);
  cmac_conj(acc, U.u[6 + i], v[2]);
  return acc;
}
template <class R>
QCU_D void su3_mul(Cplx<R> o[3], const Link<R>& U, const Cplx<R> v[3]) {
#pragma unroll
  for (int i = 0; i < 3; i++) o[i] = su3_row(U, v, i);
}
template <class R>
QCU_D void su3_dag_mul(Cplx<R> o[3], const Link<R>& U, const Cplx<R> v[3]) {
#pragma unroll
  for (int i = 0; i < 3; i++) o[i] = su3_dag_row(U, v, i);
}

// out += reconstruct(U h) (FWD) or reconstruct(U^dag h). ROWS: each colour row
// of the products is added in as soon as it is formed (fewer live registers;
// the same operations): faster for batched FP64 launches at a 128-register
// cap, slower for single-RHS ones without a cap.
template <int MU, bool FWD, int F, bool ROWS, class R>
QCU_D void mul_reconstruct(Spinor<R>& o, const Link<R>& U, const Half2<R>& h) {
  if constexpr (ROWS) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const Cplx<R> a = FWD ? su3_row(U, h.h0, i) : su3_dag_row(U, h.h0, i);
      const Cplx<R> b = FWD ? su3_row(U, h.h1, i) : su3_dag_row(U, h.h1, i);
      reconstruct_row<MU, FWD, F>(o, i, a, b);
    }
  } else {
    Cplx<R> a[3], b[3];
    if (FWD) {
      su3_mul(a, U, h.h0);
      su3_mul(b, U, h.h1);
    } else {
      su3_dag_mul(a, U, h.h0);
      su3_dag_mul(b, U, h.h1);
    }
    reconstruct<MU, FWD, F>(o, a, b);
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
template <int PS, int PL, int MU, int F, bool ROWS, class R>
QCU_D void hop_dir(Spinor<R>& o, const Geom& g, const Nbrs& nb, int parity, int s, int r,
                   const CSpinorView& in, const void* gauge, R bc_t) {
  Link<R> U;
  Half2<R> h;
  // forward: U_mu(x) in(x+mu)
  LinkIO<PL>::load(U, gauge, g.Vh_pad, MU, parity, s);
  load_project<PS, MU, true, F>(h, in, nb.fwd[MU], r, (MU == 3 && nb.tf) ? bc_t : R(1));
  mul_reconstruct<MU, true, F, ROWS>(o, U, h);
  // backward: U_mu(x-mu)^dag in(x-mu); the link lives on the other parity
  LinkIO<PL>::load(U, gauge, g.Vh_pad, MU, 1 - parity, nb.bwd[MU]);
  load_project<PS, MU, false, F>(h, in, nb.bwd[MU], r, (MU == 3 && nb.tb) ? bc_t : R(1));
  mul_reconstruct<MU, false, F, ROWS>(o, U, h);
}

// ---------------------------------------------------------------------------
// 16-bit spinors: the hop in paired FP32 instructions (sm_100 FFMA2/FADD2/
// FMUL2). Two-component spin vectors are kept "spin-paired": lane 0 holds the
// upper component (h0, or spin 0 / spin 2 of the output), lane 1 the lower
// (h1, or spin 1 / spin 3), with real and imaginary parts in separate pairs.
// One SU(3) multiply then serves both half-spinor components, and the
// projection, scaling and reconstruction act on two components per
// instruction. The 16-bit decode writes the neighbour's components straight
// into the pairs each direction needs. Same arithmetic as the scalar path per
// component (sums may associate differently).
// ---------------------------------------------------------------------------
struct HalfPair {
  float2 re[3], im[3];
};

// Spin-paired accumulator: U = (o0, o1), L = (o2, o3), X = (o3, o2): the
// directions whose reconstruction pairs the lower spins in swapped order (0
// and 1) add into X, which is folded into L before directions 2 and 3.
struct SpinPair {
  float2 ure[3], uim[3], lre[3], lim[3], xre[3], xim[3];
};

// integer-valued 16-bit components of words a and b as a pair (offset removed
// by one paired add)
QCU_D float2 dec_lo2(int a, int b) {
  return fadd2(make_float2(u16f(a, 0x7410), u16f(b, 0x7410)), splat2(-8421376.0f));
}
QCU_D float2 dec_hi2(int a, int b) {
  return fadd2(make_float2(u16f(a, 0x7432), u16f(b, 0x7432)), splat2(-8421376.0f));
}
// The raw 16-bit values of words a (lane 0) and b (lane 1), low or high
// halves: 8421376 + v, integers in [2^23, 2^24).
QCU_D float2 raw_lo2(int a, int b) { return make_float2(u16f(a, 0x7410), u16f(b, 0x7410)); }
QCU_D float2 raw_hi2(int a, int b) { return make_float2(u16f(a, 0x7432), u16f(b, 0x7432)); }
// p + s q per lane (s = S0, S1 = +-1) of raw values p and q, exactly, which
// equals dec(p) + s dec(q): where s = -1 the offsets cancel in the difference
// of two integers in [2^23, 2^24); where s = +1 twice the offset comes off p
// first (an integer below 2^24 in magnitude) and q's offset restores one.
// One or two paired instructions instead of the decode's two and the
// combination's one.
template <int S0, int S1>
QCU_D float2 raw_comb2(float2 p, float2 q) {
  if constexpr (S0 < 0 && S1 < 0) {
    return ffma2(q, splat2(-1.f), p);
  } else {
    constexpr float c0 = S0 > 0 ? -16842752.0f : 0.f, c1 = S1 > 0 ? -16842752.0f : 0.f;
    return ffma2(q, make_float2((float)S0, (float)S1), fadd2(p, make_float2(c0, c1)));
  }
}
QCU_D int word_of(const int4 w[3], int k) {
  const int4 c = w[k >> 2];
  const int l = k & 3;
  return l == 0 ? c.x : (l == 1 ? c.y : (l == 2 ? c.z : c.w));
}

// 16-bit 12-real links in units of the 16-bit grid: rows 0 and 1 decoded two
// entries per paired subtraction, row 2 = conj(row0 x row1) / 32767 in the
// same units (the stencil scales the product by 1/32767 per neighbour).
template <> struct LinkIO<LINK_HALF_RAW> {
  typedef float R;
  static QCU_D void load(Link<R>& L, const void* gauge, int Vh_pad, int mu, int parity, int s) {
    const int2* p = static_cast<const int2*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 3;
    int2 w[3];
#pragma unroll
    for (int c = 0; c < 3; c++) w[c] = __ldg(p + chunk_index(c, s, 0, 3, 1));
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2 re = dec_lo2(w[c].x, w[c].y), im = dec_hi2(w[c].x, w[c].y);
      L.u[2 * c] = mk(re.x, im.x);
      L.u[2 * c + 1] = mk(re.y, im.y);
    }
    su3_reconstruct(L);
#pragma unroll
    for (int k = 6; k < 9; k++) L.u[k] = kInvFix * L.u[k];
  }
};
// the factor that converts a link of format PL to its value
template <int PL> QCU_HD constexpr float link_unit() { return PL == LINK_HALF_RAW ? kInvFix : 1.f; }

// h = P_mu psi of the 16-bit neighbour spinor, spin-paired, in units of its
// 16-bit grid; returns the scale (norm times `phase`) that the reconstruction
// applies (the hop is linear, so scaling U h equals scaling h). Same projector
// rows as project().
template <int MU, bool FWD, int F>
QCU_D float load_project_pair(HalfPair& h, const CSpinorView& in, int s, int r, float phase) {
  constexpr int S = FWD ? -F : F;
  constexpr bool SWAP = (MU == 0 || MU == 1);  // lower pair as (p3, p2)
  const int4* p = static_cast<const int4*>(in.data);
  int4 w[3];
#pragma unroll
  for (int c = 0; c < 3; c++) w[c] = p[chunk_index(c, s, r, 3, in.nrhs)];
  const float nm = in.norm[site_rhs_index(s, r, in.nrhs)] * kInvFix * phase;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    // component k = 3*spin + colour; word k holds (re, im) as (lo, hi)
    const int w0 = word_of(w, c), w1 = word_of(w, 3 + c);
    const int w2 = word_of(w, SWAP ? 9 + c : 6 + c), w3 = word_of(w, SWAP ? 6 + c : 9 + c);
    // raw values; the combinations below are exact, as with decoded values
    const float2 Pre = raw_lo2(w0, w1), Pim = raw_hi2(w0, w1);
    const float2 Qre = raw_lo2(w2, w3), Qim = raw_hi2(w2, w3);
    float2 hre, him;
    if constexpr (MU == 0) {  // h0 = p0 + S i p3, h1 = p1 + S i p2; Q = (p3, p2)
      hre = raw_comb2<-S, -S>(Pre, Qim);
      him = raw_comb2<S, S>(Pim, Qre);
    } else if constexpr (MU == 1) {  // h0 = p0 - S p3, h1 = p1 + S p2; Q = (p3, p2)
      hre = raw_comb2<-S, S>(Pre, Qre);
      him = raw_comb2<-S, S>(Pim, Qim);
    } else if constexpr (MU == 2) {  // h0 = p0 + S i p2, h1 = p1 - S i p3; Q = (p2, p3)
      hre = raw_comb2<-S, S>(Pre, Qim);
      him = raw_comb2<S, -S>(Pim, Qre);
    } else {  // h0 = p0 + S p2, h1 = p1 + S p3; Q = (p2, p3)
      hre = raw_comb2<S, S>(Pre, Qre);
      him = raw_comb2<S, S>(Pim, Qim);
    }
    h.re[c] = hre;
    h.im[c] = him;
  }
  return nm;
}

// row i of a = U h (FWD) or U^dag h, both spin components at once
template <bool FWD>
QCU_D void su3_row_pair(float2& re, float2& im, const Link<float>& U, const HalfPair& h, int i) {
  re = make_float2(0.f, 0.f);
  im = make_float2(0.f, 0.f);
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const Cplx<float> u = FWD ? U.u[i * 3 + j] : U.u[j * 3 + i];
    const float2 ur = splat2(u.re), ui = splat2(u.im);
    if (FWD) {  // u h
      re = ffma2(ur, h.re[j], re);
      re = ffma2(fneg2(ui), h.im[j], re);
      im = ffma2(ur, h.im[j], im);
      im = ffma2(ui, h.re[j], im);
    } else {  // conj(u) h
      re = ffma2(ur, h.re[j], re);
      re = ffma2(ui, h.im[j], re);
      im = ffma2(ur, h.im[j], im);
      im = ffma2(fneg2(ui), h.re[j], im);
    }
  }
}

// out += sc * reconstruct(U h) (or U^dag h), spin-paired (lanes: from h0,
// from h1); same rows as reconstruct(), with the neighbour's scale folded
// into the sign factors. Each colour row of the product is added in as soon
// as it is formed, so only one row is live at a time.
template <int MU, bool FWD, int F>
QCU_D void mul_reconstruct_pair(SpinPair& o, const Link<float>& U, const HalfPair& h, float sc) {
  constexpr int S = FWD ? -F : F;
  const float fS = (float)S * sc;
  const float2 up = splat2(sc);
  const float2 same = splat2(fS), nsame = splat2(-fS);
  const float2 mixed = make_float2(-fS, fS), mixed_r = make_float2(fS, -fS);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float2 are, aim;
    su3_row_pair<FWD>(are, aim, U, h, c);
    o.ure[c] = ffma2(are, up, o.ure[c]);
    o.uim[c] = ffma2(aim, up, o.uim[c]);
    if constexpr (MU == 0) {  // o2 -= S i b, o3 -= S i a  ->  X = (o3, o2) -= S i (a, b)
      o.xre[c] = ffma2(aim, same, o.xre[c]);
      o.xim[c] = ffma2(are, nsame, o.xim[c]);
    } else if constexpr (MU == 1) {  // o2 += S b, o3 -= S a  ->  X += (-S a, S b)
      o.xre[c] = ffma2(are, mixed, o.xre[c]);
      o.xim[c] = ffma2(aim, mixed, o.xim[c]);
    } else if constexpr (MU == 2) {  // o2 -= S i a, o3 += S i b  ->  L += (-S i a, S i b)
      o.lre[c] = ffma2(aim, mixed_r, o.lre[c]);
      o.lim[c] = ffma2(are, mixed, o.lim[c]);
    } else {  // o2 += S a, o3 += S b
      o.lre[c] = ffma2(are, same, o.lre[c]);
      o.lim[c] = ffma2(aim, same, o.lim[c]);
    }
  }
}

template <int PL, int MU, int F>
QCU_D void hop_dir_pair(SpinPair& o, const Geom& g, const Nbrs& nb, int parity, int s, int r, const CSpinorView& in,
                        const void* gauge, float bc_t) {
  Link<float> U;
  HalfPair h;
  constexpr float unit = link_unit<PL>();
  LinkIO<PL>::load(U, gauge, g.Vh_pad, MU, parity, s);
  float sc = load_project_pair<MU, true, F>(h, in, nb.fwd[MU], r, (MU == 3 && nb.tf) ? bc_t * unit : unit);
  mul_reconstruct_pair<MU, true, F>(o, U, h, sc);
  LinkIO<PL>::load(U, gauge, g.Vh_pad, MU, 1 - parity, nb.bwd[MU]);
  sc = load_project_pair<MU, false, F>(h, in, nb.bwd[MU], r, (MU == 3 && nb.tb) ? bc_t * unit : unit);
  mul_reconstruct_pair<MU, false, F>(o, U, h, sc);
}

template <int PL, bool DAG>
QCU_D void hop_spin_pair(SpinPair& o, const Geom& g, int parity, int s, int r, const CSpinorView& in,
                         const void* gauge, float bc_t) {
  constexpr int F = DAG ? -1 : 1;
#pragma unroll
  for (int c = 0; c < 3; c++) o.ure[c] = o.uim[c] = o.xre[c] = o.xim[c] = make_float2(0.f, 0.f);
  const Nbrs nb = neighbours(g, s, parity);
  hop_dir_pair<PL, 0, F>(o, g, nb, parity, s, r, in, gauge, bc_t);
  hop_dir_pair<PL, 1, F>(o, g, nb, parity, s, r, in, gauge, bc_t);
  // only directions 0 and 1 add into X, only 2 and 3 into L: fold X into L
  // now, so that the second half of the hop holds one lower accumulator
#pragma unroll
  for (int c = 0; c < 3; c++) {
    o.lre[c] = make_float2(o.xre[c].y, o.xre[c].x);
    o.lim[c] = make_float2(o.xim[c].y, o.xim[c].x);
  }
  hop_dir_pair<PL, 2, F>(o, g, nb, parity, s, r, in, gauge, bc_t);
  hop_dir_pair<PL, 3, F>(o, g, nb, parity, s, r, in, gauge, bc_t);
}

template <int PL, bool DAG>
QCU_D void hop_half_pair(Spinor<float>& out, const Geom& g, int parity, int s, int r, const CSpinorView& in,
                         const void* gauge, float bc_t) {
  SpinPair o;
  hop_spin_pair<PL, DAG>(o, g, parity, s, r, in, gauge, bc_t);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    out.c[c] = mk(o.ure[c].x, o.uim[c].x);
    out.c[3 + c] = mk(o.ure[c].y, o.uim[c].y);
    out.c[6 + c] = mk(o.lre[c].x, o.lim[c].x);
    out.c[9 + c] = mk(o.lre[c].y, o.lim[c].y);
  }
}

// ---------------------------------------------------------------------------
// Block-paired spinors for the fast 16-bit operator's epilogues: pair j holds
// component j of chiral block 0 (spins 0,1) in lane 0 and component j of
// block 1 (spins 2,3) in lane 1, i.e. (c[j], c[6+j]). The two 6x6 clover
// blocks then multiply both halves of the spinor in one paired instruction
// each, with the block-interleaved FP32 clover supplying matching pairs, and
// xpay, the 16-bit decode and encode and the norm stay paired too.
// ---------------------------------------------------------------------------
struct SpinBlock {
  float2 re[6], im[6];
};

template <int PL, bool DAG>
QCU_D void hop_half_block(SpinBlock& out, const Geom& g, int parity, int s, int r, const CSpinorView& in,
                          const void* gauge, float bc_t) {
  SpinPair o;
  hop_spin_pair<PL, DAG>(o, g, parity, s, r, in, gauge, bc_t);
#pragma unroll
  for (int c = 0; c < 3; c++) {  // spin 0 and 2 of colour c, then spin 1 and 3
    out.re[c] = make_float2(o.ure[c].x, o.lre[c].x);
    out.im[c] = make_float2(o.uim[c].x, o.lim[c].x);
    out.re[3 + c] = make_float2(o.ure[c].y, o.lre[c].y);
    out.im[3 + c] = make_float2(o.uim[c].y, o.lim[c].y);
  }
}

// v <- blockdiag(B0, B1) v, FP32 block-interleaved clover
QCU_D void clover_apply_block(SpinBlock& v, const void* clov, int Vh_pad, int parity, int s) {
  const float4* p = static_cast<const float4*>(clov) + (size_t)parity * Vh_pad * 18;
  float2 ore[6], oim[6];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const float4 w = __ldg(p + chunk_index(q, s, 0, 18, 1));
    const float2 d0 = make_float2(w.x, w.y), d1 = make_float2(w.z, w.w);
    ore[2 * q] = fmul2(d0, v.re[2 * q]);
    oim[2 * q] = fmul2(d0, v.im[2 * q]);
    ore[2 * q + 1] = fmul2(d1, v.re[2 * q + 1]);
    oim[2 * q + 1] = fmul2(d1, v.im[2 * q + 1]);
  }
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++) {
      const float4 w = __ldg(p + chunk_index(3 + tri_index(i, j), s, 0, 18, 1));
      const float2 mre = make_float2(w.x, w.y), mim = make_float2(w.z, w.w);
      // o_i += M_ij v_j ; o_j += conj(M_ij) v_i
      ore[i] = ffma2(mre, v.re[j], ore[i]);
      ore[i] = ffma2(fneg2(mim), v.im[j], ore[i]);
      oim[i] = ffma2(mre, v.im[j], oim[i]);
      oim[i] = ffma2(mim, v.re[j], oim[i]);
      ore[j] = ffma2(mre, v.re[i], ore[j]);
      ore[j] = ffma2(mim, v.im[i], ore[j]);
      oim[j] = ffma2(mre, v.im[i], oim[j]);
      oim[j] = ffma2(fneg2(mim), v.re[i], oim[j]);
    }
#pragma unroll
  for (int j = 0; j < 6; j++) {
    v.re[j] = ore[j];
    v.im[j] = oim[j];
  }
}

// v <- blockdiag(B0, B1) v, 16-bit clover (CloverIO<PREC_HALF>: per site 36
// words, block b's element word k at word 18b + k, and one norm): the words of
// the two blocks decode into the lanes of one pair, so the multiply is the
// one of clover_apply_block; the site's scale (norm / 32767) is applied to
// the result.
QCU_D void clover_apply_block16(SpinBlock& v, const void* clov, int Vh_pad, int parity, int s) {
  const int4* p = static_cast<const int4*>(clov) + (size_t)parity * Vh_pad * 9;
  int4 c[9];
#pragma unroll
  for (int q = 0; q < 9; q++) c[q] = __ldg(p + chunk_index(q, s, 0, 9, 1));
  const float nm = __ldg(CloverIO<PREC_HALF>::norms(clov, Vh_pad) + (size_t)parity * Vh_pad + s) * kInvFix;
  auto w = [&](int k) { return CloverIO<PREC_HALF>::word(c, k); };
  float2 ore[6], oim[6];
#pragma unroll
  for (int q = 0; q < 3; q++) {  // diagonal words: (d_2q, d_2q+1) of each block
    const float2 d0 = dec_lo2(w(q), w(18 + q)), d1 = dec_hi2(w(q), w(18 + q));
    ore[2 * q] = fmul2(d0, v.re[2 * q]);
    oim[2 * q] = fmul2(d0, v.im[2 * q]);
    ore[2 * q + 1] = fmul2(d1, v.re[2 * q + 1]);
    oim[2 * q + 1] = fmul2(d1, v.im[2 * q + 1]);
  }
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++) {
      const int k = 3 + tri_index(i, j);
      const float2 mre = dec_lo2(w(k), w(18 + k)), mim = dec_hi2(w(k), w(18 + k));
      ore[i] = ffma2(mre, v.re[j], ore[i]);
      ore[i] = ffma2(fneg2(mim), v.im[j], ore[i]);
      oim[i] = ffma2(mre, v.im[j], oim[i]);
      oim[i] = ffma2(mim, v.re[j], oim[i]);
      ore[j] = ffma2(mre, v.re[i], ore[j]);
      ore[j] = ffma2(mim, v.im[i], ore[j]);
      oim[j] = ffma2(mre, v.im[i], oim[j]);
      oim[j] = ffma2(fneg2(mim), v.re[i], oim[j]);
    }
#pragma unroll
  for (int j = 0; j < 6; j++) {
    v.re[j] = fmul2(ore[j], splat2(nm));
    v.im[j] = fmul2(oim[j], splat2(nm));
  }
}

QCU_D void load16_block(SpinBlock& v, const CSpinorView& f, int s, int r) {
  const int4* p = static_cast<const int4*>(f.data);
  int4 w[3];
#pragma unroll
  for (int c = 0; c < 3; c++) w[c] = p[chunk_index(c, s, r, 3, f.nrhs)];
  const float2 nm = splat2(f.norm[site_rhs_index(s, r, f.nrhs)] * kInvFix);
#pragma unroll
  for (int j = 0; j < 6; j++) {
    const int a = word_of(w, j), b = word_of(w, 6 + j);
    v.re[j] = fmul2(dec_lo2(a, b), nm);
    v.im[j] = fmul2(dec_hi2(a, b), nm);
  }
}

QCU_D void store16_block(const SpinorView& f, int s, int r, const SpinBlock& v) {
  float mx = 0.f;
#pragma unroll
  for (int j = 0; j < 6; j++)
    mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.re[j].x), fabsf(v.re[j].y)), fmaxf(fabsf(v.im[j].x), fabsf(v.im[j].y))));
  const float sc = mx > 0.f ? kFix / mx : 0.f;
  float2 tre[6], tim[6];
#pragma unroll
  for (int j = 0; j < 6; j++) {  // the roundings of pack16(x * sc, ...)
    tre[j] = fadd2(fmul2(v.re[j], splat2(sc)), splat2(8421376.0f));
    tim[j] = fadd2(fmul2(v.im[j], splat2(sc)), splat2(8421376.0f));
  }
  int words[12];
#pragma unroll
  for (int j = 0; j < 6; j++) {
    words[j] = (int)__byte_perm(__float_as_uint(tre[j].x), __float_as_uint(tim[j].x), 0x5410);
    words[6 + j] = (int)__byte_perm(__float_as_uint(tre[j].y), __float_as_uint(tim[j].y), 0x5410);
  }
  int4* p = static_cast<int4*>(f.data);
#pragma unroll
  for (int c = 0; c < 3; c++)
    p[chunk_index(c, s, r, 3, f.nrhs)] = make_int4(words[4 * c], words[4 * c + 1], words[4 * c + 2], words[4 * c + 3]);
  f.norm[site_rhs_index(s, r, f.nrhs)] = mx;
}

// |v|^2, summed in FP32 pairs (the sloppy solver's dot products)
QCU_D float norm2_block(const SpinBlock& v) {
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll
  for (int j = 0; j < 6; j++) {
    acc = ffma2(v.re[j], v.re[j], acc);
    acc = ffma2(v.im[j], v.im[j], acc);
  }
  return acc.x + acc.y;
}

// component k (= spin*3 + colour) of a block-paired spinor
QCU_D Cplx<float> block_comp(const SpinBlock& v, int k) {
  return k < 6 ? mk(v.re[k].x, v.im[k].x) : mk(v.re[k - 6].y, v.im[k - 6].y);
}

template <int PS, int PL, bool DAG, bool ROWS = false, class R>
QCU_D void hop(Spinor<R>& o, const Geom& g, int parity, int s, int r, const CSpinorView& in,
               const void* gauge, R bc_t) {
// Paired-FP32 hop for 16-bit spinors (1, default) or the scalar one (0).
// Measured on B200 at 32^4 with 16 RHS: hop 677 vs 733 us.
#ifndef QCU_HOP_FFMA2
#define QCU_HOP_FFMA2 1
#endif
  if constexpr (PS == PREC_HALF && QCU_HOP_FFMA2) {
    hop_half_pair<PL, DAG>(o, g, parity, s, r, in, gauge, bc_t);
    return;
  }
  constexpr int F = DAG ? -1 : 1;
#pragma unroll
  for (int k = 0; k < 12; k++) o.c[k] = mk(R(0), R(0));
  const Nbrs nb = neighbours(g, s, parity);
  hop_dir<PS, PL, 0, F, ROWS>(o, g, nb, parity, s, r, in, gauge, bc_t);
  hop_dir<PS, PL, 1, F, ROWS>(o, g, nb, parity, s, r, in, gauge, bc_t);
  hop_dir<PS, PL, 2, F, ROWS>(o, g, nb, parity, s, r, in, gauge, bc_t);
  hop_dir<PS, PL, 3, F, ROWS>(o, g, nb, parity, s, r, in, gauge, bc_t);
}

}  // namespace qcu
