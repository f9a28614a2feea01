// RHS-paired stencil bodies for batched launches of the fast 16-bit operator
// (16-bit spinors, FP32 18-real links, FP32 block-interleaved clover).
//
// One thread serves one site and two adjacent right-hand sides r, r+1, which
// occupy the two lanes of paired FP32 instructions (sm_100 FFMA2/FADD2/FMUL2):
// every component of the spinor is a (lane r, lane r+1) pair for its real and
// one for its imaginary part. The link, the clover block, the neighbour
// indices and the addresses are then formed once for two right-hand sides,
// and every multiply by a link or clover element is one paired instruction
// for both. Per lane the arithmetic is the same sequence of roundings as the
// one-RHS-per-thread kernels (spin-paired hop, herm_apply, pack16), so a
// column's result does not depend on which column shares its thread.
#pragma once
#include "qcu_dslash.cuh"
#include "qcu_kernels.cuh"
#include "qcu_reduce.cuh"

namespace qcu {

// component k = 3*spin + colour; lane 0 = RHS r, lane 1 = RHS r+1
struct PairSpinor {
  float2 re[12], im[12];
};

// The two RHS lanes of a thread: r0 and r1 = r0 + d (d = 0 when r0 is the
// last column of an odd batch; lane 1 then repeats lane 0 and is not stored).
struct RhsPair {
  int r0, d;
};

// both lanes' 16-bit chunks of site s: w0 (lane 0) and w1 (lane 1); returns
// the lanes' norms
QCU_D float2 load_words_pair(int4 w0[3], int4 w1[3], const CSpinorView& f, int s, RhsPair rp) {
  const int4* p = static_cast<const int4*>(f.data);
  const unsigned i0 = (unsigned)chunk_index(0, s, rp.r0, 3, f.nrhs);
  const unsigned cs = 32u * (unsigned)f.nrhs;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    w0[c] = p[i0 + c * cs];
    w1[c] = p[i0 + c * cs + rp.d];
  }
  const unsigned n0 = (unsigned)site_rhs_index(s, rp.r0, f.nrhs);
  return make_float2(f.norm[n0], f.norm[n0 + rp.d]);
}

// h = P_mu psi of the neighbour, both lanes, in units of the 16-bit grid, and
// the scale (norm x phase) the reconstruction applies. Same projector rows as
// load_project_pair.
template <int MU, bool FWD, int F>
QCU_D float2 project_rp(float2 h0re[3], float2 h0im[3], float2 h1re[3], float2 h1im[3], const int4 w0[3],
                        const int4 w1[3], float2 nm, float phase) {
  constexpr int S = FWD ? -F : F;
  const float2 sc = fmul2(nm, splat2(kInvFix * phase));
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float2 pre[4], pim[4];  // raw values (raw_comb2 combines them exactly)
#pragma unroll
    for (int sp = 0; sp < 4; sp++) {
      const int a = word_of(w0, 3 * sp + c), b = word_of(w1, 3 * sp + c);
      pre[sp] = raw_lo2(a, b);
      pim[sp] = raw_hi2(a, b);
    }
    if constexpr (MU == 0) {  // h0 = p0 + S i p3, h1 = p1 + S i p2
      h0re[c] = raw_comb2<-S, -S>(pre[0], pim[3]);
      h0im[c] = raw_comb2<S, S>(pim[0], pre[3]);
      h1re[c] = raw_comb2<-S, -S>(pre[1], pim[2]);
      h1im[c] = raw_comb2<S, S>(pim[1], pre[2]);
    } else if constexpr (MU == 1) {  // h0 = p0 - S p3, h1 = p1 + S p2
      h0re[c] = raw_comb2<-S, -S>(pre[0], pre[3]);
      h0im[c] = raw_comb2<-S, -S>(pim[0], pim[3]);
      h1re[c] = raw_comb2<S, S>(pre[1], pre[2]);
      h1im[c] = raw_comb2<S, S>(pim[1], pim[2]);
    } else if constexpr (MU == 2) {  // h0 = p0 + S i p2, h1 = p1 - S i p3
      h0re[c] = raw_comb2<-S, -S>(pre[0], pim[2]);
      h0im[c] = raw_comb2<S, S>(pim[0], pre[2]);
      h1re[c] = raw_comb2<S, S>(pre[1], pim[3]);
      h1im[c] = raw_comb2<-S, -S>(pim[1], pre[3]);
    } else {  // h0 = p0 + S p2, h1 = p1 + S p3
      h0re[c] = raw_comb2<S, S>(pre[0], pre[2]);
      h0im[c] = raw_comb2<S, S>(pim[0], pim[2]);
      h1re[c] = raw_comb2<S, S>(pre[1], pre[3]);
      h1im[c] = raw_comb2<S, S>(pim[1], pim[3]);
    }
  }
  return sc;
}

// ---------------------------------------------------------------------------
// Staged neighbour words. At its start each thread copies the words and norms
// of its far neighbours (t; or z and t) for both lanes into its own slots of
// shared memory with cp.async, computes the other hops from global memory
// meanwhile, waits for its own copies and reads those hops from its slots:
// the far neighbours' loads are in flight from the start without holding
// registers. Slot set k (fwd, bwd of each staged direction): words
// [k][chunk][lane][thread], norms [k][lane][thread], so a warp's accesses are
// consecutive 16- or 4-byte words.
// ---------------------------------------------------------------------------
extern __shared__ int4 qcu_staged[];  // dynamic shared memory of the staged kernels

// NT slot sets of the block's threads
template <int NT>
struct StagedTiles {
  int tid, nth;  // thread of the block, threads of the block
  QCU_D int4* w(int k, int j) const { return qcu_staged + (k * 6 + j) * nth + tid; }
  QCU_D float* n(int k, int lane) const {
    return reinterpret_cast<float*>(qcu_staged + NT * 6 * nth) + (k * 2 + lane) * nth + tid;
  }
};

QCU_D void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
QCU_D void cp_async4(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
QCU_D void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// both lanes' words and norms of site sn into the thread's slot set k
template <int NT>
QCU_D void stage_site(const StagedTiles<NT>& T, int k, const CSpinorView& f, int sn, RhsPair rp) {
  const int4* p = static_cast<const int4*>(f.data);
  const unsigned i0 = (unsigned)chunk_index(0, sn, rp.r0, 3, f.nrhs);
  const unsigned cs = 32u * (unsigned)f.nrhs;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    cp_async16(T.w(k, 2 * c), p + i0 + c * cs);
    cp_async16(T.w(k, 2 * c + 1), p + i0 + c * cs + rp.d);
  }
  const unsigned n0 = (unsigned)site_rhs_index(sn, rp.r0, f.nrhs);
  cp_async4(T.n(k, 0), f.norm + n0);
  cp_async4(T.n(k, 1), f.norm + n0 + rp.d);
}

// both lanes' words of the thread's slot set k; returns the norms
template <int NT>
QCU_D float2 load_words_staged(int4 w0[3], int4 w1[3], const StagedTiles<NT>& T, int k) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    w0[c] = *T.w(k, 2 * c);
    w1[c] = *T.w(k, 2 * c + 1);
  }
  return make_float2(*T.n(k, 0), *T.n(k, 1));
}

// row i of U h (FWD) or U^dag h for one half-spinor component, both lanes;
// the order of the multiply-adds is that of su3_row_pair
template <bool FWD>
QCU_D void su3_row_rp(float2& re, float2& im, const Link<float>& U, const float2 hre[3], const float2 him[3], int i) {
  re = make_float2(0.f, 0.f);
  im = make_float2(0.f, 0.f);
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const Cplx<float> u = FWD ? U.u[i * 3 + j] : U.u[j * 3 + i];
    const float2 ur = splat2(u.re), ui = splat2(u.im);
    if (FWD) {
      re = ffma2(ur, hre[j], re);
      re = ffma2(fneg2(ui), him[j], re);
      im = ffma2(ur, him[j], im);
      im = ffma2(ui, hre[j], im);
    } else {
      re = ffma2(ur, hre[j], re);
      re = ffma2(ui, him[j], re);
      im = ffma2(ur, him[j], im);
      im = ffma2(fneg2(ui), hre[j], im);
    }
  }
}

// o += sc * reconstruct(U h): spins 0 and 1 take a = U h0 and b = U h1, spins
// 2 and 3 the rows of reconstruct() with the sign folded into the scale
template <int MU, bool FWD, int F>
QCU_D void mul_reconstruct_rp(PairSpinor& o, const Link<float>& U, const float2 h0re[3], const float2 h0im[3],
                              const float2 h1re[3], const float2 h1im[3], float2 sc) {
  constexpr int S = FWD ? -F : F;
  const float2 sp = fmul2(sc, splat2((float)S)), sn = fmul2(sc, splat2((float)-S));
#pragma unroll
  for (int i = 0; i < 3; i++) {
    float2 are, aim, bre, bim;
    su3_row_rp<FWD>(are, aim, U, h0re, h0im, i);
    su3_row_rp<FWD>(bre, bim, U, h1re, h1im, i);
    o.re[i] = ffma2(are, sc, o.re[i]);
    o.im[i] = ffma2(aim, sc, o.im[i]);
    o.re[3 + i] = ffma2(bre, sc, o.re[3 + i]);
    o.im[3 + i] = ffma2(bim, sc, o.im[3 + i]);
    float2 &o2re = o.re[6 + i], &o2im = o.im[6 + i], &o3re = o.re[9 + i], &o3im = o.im[9 + i];
    if constexpr (MU == 0) {  // o2 -= S i b, o3 -= S i a
      o2re = ffma2(bim, sp, o2re);
      o2im = ffma2(bre, sn, o2im);
      o3re = ffma2(aim, sp, o3re);
      o3im = ffma2(are, sn, o3im);
    } else if constexpr (MU == 1) {  // o2 += S b, o3 -= S a
      o2re = ffma2(bre, sp, o2re);
      o2im = ffma2(bim, sp, o2im);
      o3re = ffma2(are, sn, o3re);
      o3im = ffma2(aim, sn, o3im);
    } else if constexpr (MU == 2) {  // o2 -= S i a, o3 += S i b
      o2re = ffma2(aim, sp, o2re);
      o2im = ffma2(are, sn, o2im);
      o3re = ffma2(bim, sn, o3re);
      o3im = ffma2(bre, sp, o3im);
    } else {  // o2 += S a, o3 += S b
      o2re = ffma2(are, sp, o2re);
      o2im = ffma2(aim, sp, o2im);
      o3re = ffma2(bre, sp, o3re);
      o3im = ffma2(bim, sp, o3im);
    }
  }
}

// Both hops of direction MU. kst >= 0: the neighbours' words come from the
// thread's staged slots kst (forward) and kst + 1 (backward)
template <int MU, int F, int NT = 2>
QCU_D void hop_dir_rp(PairSpinor& o, const Geom& g, const Nbrs& nb, int parity, int s, RhsPair rp,
                      const CSpinorView& in, const void* gauge, float bc_t, const StagedTiles<NT>* T = nullptr,
                      int kst = -1) {
  Link<float> U;
  int4 w0[3], w1[3];
  float2 h0re[3], h0im[3], h1re[3], h1im[3];
  LinkIO<LINK_SINGLE18>::load(U, gauge, g.Vh_pad, MU, parity, s);
  float2 nm = kst >= 0 ? load_words_staged(w0, w1, *T, kst) : load_words_pair(w0, w1, in, nb.fwd[MU], rp);
  float2 sc = project_rp<MU, true, F>(h0re, h0im, h1re, h1im, w0, w1, nm, (MU == 3 && nb.tf) ? bc_t : 1.f);
  mul_reconstruct_rp<MU, true, F>(o, U, h0re, h0im, h1re, h1im, sc);
  LinkIO<LINK_SINGLE18>::load(U, gauge, g.Vh_pad, MU, 1 - parity, nb.bwd[MU]);
  nm = kst >= 0 ? load_words_staged(w0, w1, *T, kst + 1) : load_words_pair(w0, w1, in, nb.bwd[MU], rp);
  sc = project_rp<MU, false, F>(h0re, h0im, h1re, h1im, w0, w1, nm, (MU == 3 && nb.tb) ? bc_t : 1.f);
  mul_reconstruct_rp<MU, false, F>(o, U, h0re, h0im, h1re, h1im, sc);
}

// The hop D (or D^dag) of both lanes, in the order x, y, z, t. NS > 0: the
// last NS directions read staged slots, after the thread has waited for them
// (HALF = 1: directions up to 3 - NS; HALF = 2: the rest; HALF = 0: all four
// from global memory).
template <bool DAG, int NS, int HALF>
QCU_D void hop_rp(PairSpinor& o, const Geom& g, const Nbrs& nb, int parity, int s, RhsPair rp,
                  const CSpinorView& in, const void* gauge, float bc_t,
                  const StagedTiles<2 * (NS > 0 ? NS : 1)>* T = nullptr) {
  constexpr int F = DAG ? -1 : 1;
  if constexpr (HALF != 2) {
#pragma unroll
    for (int k = 0; k < 12; k++) o.re[k] = o.im[k] = make_float2(0.f, 0.f);
  }
  constexpr int first_staged = HALF == 0 ? 4 : 4 - NS;
  if constexpr (HALF != 2) {
    hop_dir_rp<0, F>(o, g, nb, parity, s, rp, in, gauge, bc_t);
    hop_dir_rp<1, F>(o, g, nb, parity, s, rp, in, gauge, bc_t);
    if constexpr (first_staged > 2) hop_dir_rp<2, F>(o, g, nb, parity, s, rp, in, gauge, bc_t);
    if constexpr (first_staged > 3) hop_dir_rp<3, F>(o, g, nb, parity, s, rp, in, gauge, bc_t);
  }
  if constexpr (HALF == 2) {
    if constexpr (first_staged <= 2) hop_dir_rp<2, F, 2 * NS>(o, g, nb, parity, s, rp, in, gauge, bc_t, T, 0);
    hop_dir_rp<3, F, 2 * NS>(o, g, nb, parity, s, rp, in, gauge, bc_t, T, 2 * (NS - 1));
  }
}

// Element pair of the block-interleaved FP32 clover: chunk q of the lanes'
// fields holds (b0[2q], b1[2q], b0[2q+1], b1[2q+1]); E = element 2q + h of
// block b is float b + 2h of the chunk. UNI: both lanes read one field, so the
// element is one scalar for both lanes.
template <bool UNI>
struct CloverPair {
  const float4* p0;
  const float4* p1;
  bool id0, id1;  // lane without a clover term (A = 1)
  // float i of chunk q of the first lane's field. Each block loads only its
  // own two floats of a chunk: one float4 load shared by both blocks would keep
  // the other block's halves of all 18 chunks live (measured on B200, 24^3x48,
  // 48 RHS: the hop + A^-1 stencil 1.200 -> 1.159 ms, spills of the fused K2
  // 80 -> 40 bytes)
  QCU_D float one(int q, int i) const { return __ldg(reinterpret_cast<const float*>(p0 + 32 * q) + i); }
  // float i of chunk q for each lane (scalar loads straight into the pair),
  // `id` for a lane without clover
  QCU_D float2 lanes(int q, int i, float id) const {
    const float a = __ldg(reinterpret_cast<const float*>(p0 + 32 * q) + i);
    const float b = __ldg(reinterpret_cast<const float*>(p1 + 32 * q) + i);
    return make_float2(id0 ? id : a, id1 ? id : b);
  }
};

// v <- blockdiag(B0, B1) v for both lanes, block by block; per lane the order
// of herm_apply
template <bool UNI>
QCU_D void clover_apply_rp(PairSpinor& v, const CloverPair<UNI>& C) {
#pragma unroll
  for (int b = 0; b < 2; b++) {
    float2 ore[6], oim[6];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      float2 d[2];
      if constexpr (UNI) {
        d[0] = splat2(C.one(q, b));
        d[1] = splat2(C.one(q, b + 2));
      } else {
        d[0] = C.lanes(q, b, 1.f);
        d[1] = C.lanes(q, b + 2, 1.f);
      }
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int i = 2 * q + h;
        ore[i] = fmul2(d[h], v.re[6 * b + i]);
        oim[i] = fmul2(d[h], v.im[6 * b + i]);
      }
    }
#pragma unroll
    for (int i = 1; i < 6; i++)
#pragma unroll
      for (int j = 0; j < i; j++) {
        const int k = tri_index(i, j);
        float2 mre, mim;
        if constexpr (UNI) {
          mre = splat2(C.one(3 + k, b));
          mim = splat2(C.one(3 + k, b + 2));
        } else {
          mre = C.lanes(3 + k, b, 0.f);
          mim = C.lanes(3 + k, b + 2, 0.f);
        }
        const float2 vjr = v.re[6 * b + j], vji = v.im[6 * b + j];
        const float2 vir = v.re[6 * b + i], vii = v.im[6 * b + i];
        // o_i += M_ij v_j (cmac), o_j += conj(M_ij) v_i (cmac_conj)
        ore[i] = ffma2(mre, vjr, ore[i]);
        ore[i] = ffma2(fneg2(mim), vji, ore[i]);
        oim[i] = ffma2(mre, vji, oim[i]);
        oim[i] = ffma2(mim, vjr, oim[i]);
        ore[j] = ffma2(mre, vir, ore[j]);
        ore[j] = ffma2(mim, vii, ore[j]);
        oim[j] = ffma2(mre, vii, oim[j]);
        oim[j] = ffma2(fneg2(mim), vir, oim[j]);
      }
#pragma unroll
    for (int i = 0; i < 6; i++) {
      v.re[6 * b + i] = ore[i];
      v.im[6 * b + i] = oim[i];
    }
  }
}

// the lanes' clover fields at site s (parity block `parity`); nullptr = no
// clover term for that lane
QCU_D void clover_pair_apply(PairSpinor& v, const void* c0, const void* c1, int Vh_pad, int parity, int s) {
  if (!c0 && !c1) return;
  const unsigned i0 = (unsigned)chunk_index(0, s, 0, 18, 1);
  auto base = [&](const void* c) {
    return static_cast<const float4*>(c) + (size_t)parity * Vh_pad * 18 + i0;
  };
  if (c0 == c1) {
    CloverPair<true> C{base(c0), base(c0), false, false};
    clover_apply_rp<true>(v, C);
  } else {
    // a lane without clover reads the other lane's field and replaces it by
    // the identity (A = 1: the same values as skipping the multiply)
    CloverPair<false> C{base(c0 ? c0 : c1), base(c1 ? c1 : c0), c0 == nullptr, c1 == nullptr};
    clover_apply_rp<false>(v, C);
  }
}

QCU_D void load16_rp(PairSpinor& v, const CSpinorView& f, int s, RhsPair rp) {
  int4 w0[3], w1[3];
  const float2 nm = fmul2(load_words_pair(w0, w1, f, s, rp), splat2(kInvFix));
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const int a = word_of(w0, k), b = word_of(w1, k);
    v.re[k] = fmul2(dec_lo2(a, b), nm);
    v.im[k] = fmul2(dec_hi2(a, b), nm);
  }
}

// Stores the lanes whose flag is set, with the roundings of pack16(x*sc, ...),
// one 16-byte chunk of each lane at a time
QCU_D void store16_rp(const SpinorView& f, int s, RhsPair rp, const PairSpinor& v, bool w0, bool w1) {
  float m0 = 0.f, m1 = 0.f;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    m0 = fmaxf(m0, fmaxf(fabsf(v.re[k].x), fabsf(v.im[k].x)));
    m1 = fmaxf(m1, fmaxf(fabsf(v.re[k].y), fabsf(v.im[k].y)));
  }
  const float2 sc = make_float2(m0 > 0.f ? kFix / m0 : 0.f, m1 > 0.f ? kFix / m1 : 0.f);
  int4* p = static_cast<int4*>(f.data);
  const unsigned i0 = (unsigned)chunk_index(0, s, rp.r0, 3, f.nrhs);
  const unsigned cs = 32u * (unsigned)f.nrhs;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    int wa[4], wb[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int k = 4 * c + u;
      const float2 tre = fadd2(fmul2(v.re[k], sc), splat2(8421376.0f));
      const float2 tim = fadd2(fmul2(v.im[k], sc), splat2(8421376.0f));
      wa[u] = (int)__byte_perm(__float_as_uint(tre.x), __float_as_uint(tim.x), 0x5410);
      wb[u] = (int)__byte_perm(__float_as_uint(tre.y), __float_as_uint(tim.y), 0x5410);
    }
    if (w0) p[i0 + c * cs] = make_int4(wa[0], wa[1], wa[2], wa[3]);
    if (w1) p[i0 + c * cs + rp.d] = make_int4(wb[0], wb[1], wb[2], wb[3]);
  }
  const unsigned n0 = (unsigned)site_rhs_index(s, rp.r0, f.nrhs);
  if (w0) f.norm[n0] = m0;
  if (w1) f.norm[n0 + rp.d] = m1;
}

// |v|^2 of each lane in FP32, in the order of site_norm2
QCU_D float2 norm2_rp(const PairSpinor& v) {
  float2 n = make_float2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 12; k++) {
    n = ffma2(v.re[k], v.re[k], n);
    n = ffma2(v.im[k], v.im[k], n);
  }
  return n;
}

// x += alpha p, r -= alpha z for one lane, in the order of the one-RHS
// kernels, accumulators in the storage acc_prec gives (16-bit: x and r are
// re-encoded with new site norms); returns |r|^2 of the site before storage
template <int L>
QCU_D float cgxr_lane(const DslashArgs& a, int s, int r, const PairSpinor& z) {
  constexpr int PA = acc_prec(PREC_HALF);
  const float al = (float)a.alpha[r];
  Spinor<float> xv, rv, pv;
  SpinorIO<PA>::load(xv, a.xacc, s, r);
  SpinorIO<PA>::load(rv, a.racc, s, r);
  SpinorIO<PREC_HALF>::load(pv, a.pvec, s, r);
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const float zr = L ? z.re[k].y : z.re[k].x, zi = L ? z.im[k].y : z.im[k].x;
    xv.c[k].re += al * pv.c[k].re;
    xv.c[k].im += al * pv.c[k].im;
    rv.c[k].re -= al * zr;
    rv.c[k].im -= al * zi;
  }
  SpinorIO<PA>::store(a.xacc, s, r, xv);
  SpinorIO<PA>::store(a.racc, s, r, rv);
  return (float)site_norm2(rv);
}

// o <- x + c o with the 16-bit x decoded component by component
QCU_D void xpay16_rp(PairSpinor& o, const CSpinorView& f, int s, RhsPair rp, float2 c) {
  int4 w0[3], w1[3];
  const float2 nm = fmul2(load_words_pair(w0, w1, f, s, rp), splat2(kInvFix));
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const int a = word_of(w0, k), b = word_of(w1, k);
    o.re[k] = ffma2(c, o.re[k], fmul2(dec_lo2(a, b), nm));
    o.im[k] = ffma2(c, o.im[k], fmul2(dec_hi2(a, b), nm));
  }
}

// The kernel body: thread (threadIdx.x, threadIdx.y) of the block at tile
// (site tile, RHS tile) serves RHS pair 2*(RHS tile*blockDim.x + threadIdx.x)
// + {0, 1} of site (site tile)*blockDim.y + threadIdx.y. NS > 0: the hops of
// the last NS directions (t; or z and t) read neighbour words staged in the
// thread's slots of dynamic shared memory (staged_bytes(2 NS, 2 blockDim.x,
// blockDim.y) bytes).
template <int NS, bool DAG, int EPI, class Fin>
QCU_D void dslash_pair_body(const DslashArgs& a) {
  const TileCoord tc = stencil_tile(a);
  const int r0 = 2 * (tc.rhs * blockDim.x + threadIdx.x);
  const int s = stencil_site0(a, tc) + threadIdx.y;
  const bool site_ok = s < stencil_slim(a);
  const bool has1 = r0 + 1 < a.nrhs;
  const bool v0 = site_ok && r0 < a.nrhs && (a.active == nullptr || a.active[r0]);
  const bool v1 = site_ok && has1 && (a.active == nullptr || a.active[r0 + 1]);
  const RhsPair rp{r0, has1 ? 1 : 0};
  double n0 = 0.0, n1 = 0.0;
  if (v0 || v1) {
    PairSpinor o;
    const Nbrs nb = neighbours(a.g, s, a.parity);
    StagedTiles<2 * (NS > 0 ? NS : 1)> T;
    if constexpr (NS > 0) {
      T.tid = threadIdx.y * blockDim.x + threadIdx.x;
      T.nth = blockDim.x * blockDim.y;
#pragma unroll
      for (int j = 0; j < NS; j++) {
        stage_site(T, 2 * j, a.in, nb.fwd[4 - NS + j], rp);
        stage_site(T, 2 * j + 1, a.in, nb.bwd[4 - NS + j], rp);
      }
      hop_rp<DAG, NS, 1>(o, a.g, nb, a.parity, s, rp, a.in, a.gauge, (float)a.bc_t);
      cp_async_wait_all();
    }
    const int r1 = r0 + rp.d;
    if constexpr (NS > 0)
      hop_rp<DAG, NS, 2>(o, a.g, nb, a.parity, s, rp, a.in, a.gauge, (float)a.bc_t, &T);
    else
      hop_rp<DAG, 0, 0>(o, a.g, nb, a.parity, s, rp, a.in, a.gauge, (float)a.bc_t);
    const bool need_clov = (EPI & (EPI_CPRE | EPI_CX | EPI_CPOST | EPI_OUT2)) != 0;
    const void* c0 = need_clov ? clover_of(a, r0) : nullptr;
    const void* c1 = need_clov ? clover_of(a, r1) : nullptr;
    if (EPI & EPI_CPRE) clover_pair_apply(o, c0, c1, a.g.Vh_pad, a.parity, s);
    if (EPI & EPI_XPAY) {
      const float2 c = a.coef ? make_float2((float)a.coef[r0], (float)a.coef[r1]) : splat2((float)a.coef0);
      if constexpr ((EPI & EPI_CX) != 0) {
        PairSpinor xv;
        load16_rp(xv, a.x, s, rp);
        clover_pair_apply(xv, c0, c1, a.g.Vh_pad, a.parity, s);
#pragma unroll
        for (int k = 0; k < 12; k++) {
          o.re[k] = ffma2(c, o.re[k], xv.re[k]);
          o.im[k] = ffma2(c, o.im[k], xv.im[k]);
        }
      } else {
        xpay16_rp(o, a.x, s, rp, c);
      }
      if (EPI & EPI_CPOST) clover_pair_apply(o, c0, c1, a.g.Vh_pad, a.parity, s);
    }
    if constexpr ((EPI & EPI_CGXR) != 0) {
      if (v0) n0 = cgxr_lane<0>(a, s, r0, o);
      if (v1) n1 = cgxr_lane<1>(a, s, r1, o);
    } else {
      store16_rp(a.out, s, rp, o, v0, v1);
      if (EPI & EPI_NORM) {
        const float2 n = norm2_rp(o);
        n0 = v0 ? (double)n.x : 0.0;
        n1 = v1 ? (double)n.y : 0.0;
      }
    }
    if (EPI & EPI_OUT2) {
      clover_pair_apply(o, c0, c1, a.g.Vh_pad, a.parity, s);
      store16_rp(a.out2, s, rp, o, v0, v1);
    }
  }
  if (EPI & (EPI_NORM | EPI_CGXR)) {
    double v[2] = {n0, n1};
    block_reduce_finish<1, Fin, 2>(v, a.nrhs, a.red, tc);
  }
}

}  // namespace qcu
