// Loads and stores of spinors, links and packed clover blocks in the internal
// site-blocked SoA layout (chunk_index in qcu_common.cuh), for the three
// storage precisions. Arithmetic is double for PREC_DOUBLE and float otherwise.
#pragma once
#include "qcu_common.cuh"

namespace qcu {

// A view of one spinor field (one parity, nrhs right-hand sides).
struct SpinorView {
  void* data;
  float* norm;  // PREC_HALF only: one norm per (site, rhs), index s*nrhs + r
  int nrhs;
};
struct CSpinorView {
  const void* data;
  const float* norm;
  int nrhs;
  CSpinorView() = default;
  QCU_HD CSpinorView(const void* d, const float* n, int r) : data(d), norm(n), nrhs(r) {}
  QCU_HD CSpinorView(const SpinorView& v) : data(v.data), norm(v.norm), nrhs(v.nrhs) {}
};

// ---------------- spinors ----------------
template <int P> struct SpinorIO;

template <> struct SpinorIO<PREC_DOUBLE> {
  typedef double R;
  static QCU_D void load(Spinor<R>& v, const CSpinorView& f, int s, int r) {
    const double2* p = static_cast<const double2*>(f.data);
#pragma unroll
    for (int c = 0; c < 12; c++) {
      double2 w = p[chunk_index(c, s, r, 12, f.nrhs)];
      v.c[c] = mk(w.x, w.y);
    }
  }
  static QCU_D void store(const SpinorView& f, int s, int r, const Spinor<R>& v) {
    double2* p = static_cast<double2*>(f.data);
#pragma unroll
    for (int c = 0; c < 12; c++) p[chunk_index(c, s, r, 12, f.nrhs)] = make_double2(v.c[c].re, v.c[c].im);
  }
};

template <> struct SpinorIO<PREC_SINGLE> {
  typedef float R;
  static QCU_D void load(Spinor<R>& v, const CSpinorView& f, int s, int r) {
    const float4* p = static_cast<const float4*>(f.data);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      float4 w = p[chunk_index(c, s, r, 6, f.nrhs)];
      v.c[2 * c] = mk(w.x, w.y);
      v.c[2 * c + 1] = mk(w.z, w.w);
    }
  }
  static QCU_D void store(const SpinorView& f, int s, int r, const Spinor<R>& v) {
    float4* p = static_cast<float4*>(f.data);
#pragma unroll
    for (int c = 0; c < 6; c++)
      p[chunk_index(c, s, r, 6, f.nrhs)] = make_float4(v.c[2 * c].re, v.c[2 * c].im, v.c[2 * c + 1].re, v.c[2 * c + 1].im);
  }
};

// 16-bit fixed point <-> float without the conversion unit (I2F/F2I issue on
// the quarter-rate XU pipe, which bounded the 16-bit stencil). A value v in
// [-32768, 32767] is stored offset-binary, as u = v + 32768. Decoding places u
// in the mantissa of 2^23 with one byte permute (bytes u.lo, u.hi, 0x00, 0x4B),
// so the float equals 2^23 + 32768 + v and one exact subtraction recovers v.
// Encoding adds 2^23 + 32768, which rounds to the nearest integer (ties to
// even, as __float2int_rn) and leaves u in the low 16 bits of the float.
QCU_D float u16f(int w, unsigned sel) { return __uint_as_float(__byte_perm((unsigned)w, 0x4B000000u, sel)); }
QCU_D float lo16(int w) { return u16f(w, 0x7410) - 8421376.0f; }
QCU_D float hi16(int w) { return u16f(w, 0x7432) - 8421376.0f; }
QCU_D int pack16(float a, float b) {  // |a|, |b| <= 32767.49
  unsigned ia = __float_as_uint(a + 8421376.0f);
  unsigned ib = __float_as_uint(b + 8421376.0f);
  return (int)__byte_perm(ia, ib, 0x5410);
}

// Paired FP32 instructions of sm_100 (FFMA2 / FMUL2 / FADD2): two lanes per
// instruction, each lane rounded exactly as the scalar instruction.
QCU_D float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
QCU_D float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
QCU_D float2 fadd2(float2 a, float2 b) { return __fadd2_rn(a, b); }
QCU_D float2 fneg2(float2 a) { return make_float2(-a.x, -a.y); }
QCU_D float2 splat2(float a) { return make_float2(a, a); }

// (re, im) of one 16-bit word, scaled: the same roundings as lo16/hi16 times nm
QCU_D float2 dec16_pair(int w, float nm) {
  return fmul2(fadd2(make_float2(u16f(w, 0x7410), u16f(w, 0x7432)), splat2(-8421376.0f)), splat2(nm));
}
// one 16-bit word from (re, im) times sc: the same roundings as pack16(re*sc, im*sc)
QCU_D int enc16_pair(float re, float im, float sc) {
  const float2 t = fadd2(fmul2(make_float2(re, im), splat2(sc)), splat2(8421376.0f));
  return (int)__byte_perm(__float_as_uint(t.x), __float_as_uint(t.y), 0x5410);
}

template <> struct SpinorIO<PREC_HALF> {
  typedef float R;
  // integer-valued components (not yet scaled) and the factor that scales them
  static QCU_D float load_raw(Spinor<R>& v, const CSpinorView& f, int s, int r) {
    const int4* p = static_cast<const int4*>(f.data);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int4 w = p[chunk_index(c, s, r, 3, f.nrhs)];
      v.c[4 * c + 0] = mk(lo16(w.x), hi16(w.x));
      v.c[4 * c + 1] = mk(lo16(w.y), hi16(w.y));
      v.c[4 * c + 2] = mk(lo16(w.z), hi16(w.z));
      v.c[4 * c + 3] = mk(lo16(w.w), hi16(w.w));
    }
    return f.norm[site_rhs_index(s, r, f.nrhs)] * kInvFix;
  }
  static QCU_D void load(Spinor<R>& v, const CSpinorView& f, int s, int r) {
    const int4* p = static_cast<const int4*>(f.data);
    float nm = f.norm[site_rhs_index(s, r, f.nrhs)] * kInvFix;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int4 w = p[chunk_index(c, s, r, 3, f.nrhs)];
      const int ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const float2 q = dec16_pair(ws[k], nm);
        v.c[4 * c + k] = mk(q.x, q.y);
      }
    }
  }
  static QCU_D void store(const SpinorView& f, int s, int r, const Spinor<R>& v) {
    float mx = 0.f;
#pragma unroll
    for (int k = 0; k < 12; k++) mx = fmaxf(mx, fmaxf(fabsf(v.c[k].re), fabsf(v.c[k].im)));
    float sc = mx > 0.f ? kFix / mx : 0.f;
    int4* p = static_cast<int4*>(f.data);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int4 w;
      w.x = enc16_pair(v.c[4 * c + 0].re, v.c[4 * c + 0].im, sc);
      w.y = enc16_pair(v.c[4 * c + 1].re, v.c[4 * c + 1].im, sc);
      w.z = enc16_pair(v.c[4 * c + 2].re, v.c[4 * c + 2].im, sc);
      w.w = enc16_pair(v.c[4 * c + 3].re, v.c[4 * c + 3].im, sc);
      p[chunk_index(c, s, r, 3, f.nrhs)] = w;
    }
    f.norm[site_rhs_index(s, r, f.nrhs)] = mx;
  }
};

// ---------------- links ----------------
// gauge field: [dir][parity] sub-arrays of Vh_pad sites each
template <int P> struct LinkIO;

template <> struct LinkIO<PREC_DOUBLE> {
  typedef double R;
  static QCU_D void load(Link<R>& L, const void* gauge, int Vh_pad, int mu, int parity, int s) {
    const double2* p = static_cast<const double2*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 6;
#pragma unroll
    for (int c = 0; c < 6; c++) {
      double2 w = __ldg(p + chunk_index(c, s, 0, 6, 1));
      L.u[c] = mk(w.x, w.y);
    }
    su3_reconstruct(L);
  }
  static QCU_D void store(void* gauge, int Vh_pad, int mu, int parity, int s, const Link<R>& L) {
    double2* p = static_cast<double2*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 6;
#pragma unroll
    for (int c = 0; c < 6; c++) p[chunk_index(c, s, 0, 6, 1)] = make_double2(L.u[c].re, L.u[c].im);
  }
};

template <> struct LinkIO<PREC_SINGLE> {
  typedef float R;
  static QCU_D void load(Link<R>& L, const void* gauge, int Vh_pad, int mu, int parity, int s) {
    const float4* p = static_cast<const float4*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 3;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float4 w = __ldg(p + chunk_index(c, s, 0, 3, 1));
      L.u[2 * c] = mk(w.x, w.y);
      L.u[2 * c + 1] = mk(w.z, w.w);
    }
    su3_reconstruct(L);
  }
  template <class RS>
  static QCU_D void store(void* gauge, int Vh_pad, int mu, int parity, int s, const Link<RS>& L) {
    float4* p = static_cast<float4*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 3;
#pragma unroll
    for (int c = 0; c < 3; c++)
      p[chunk_index(c, s, 0, 3, 1)] = make_float4((float)L.u[2 * c].re, (float)L.u[2 * c].im,
                                                  (float)L.u[2 * c + 1].re, (float)L.u[2 * c + 1].im);
  }
};

template <> struct LinkIO<PREC_HALF> {
  typedef float R;
  static QCU_D void load(Link<R>& L, const void* gauge, int Vh_pad, int mu, int parity, int s) {
    const int2* p = static_cast<const int2*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 3;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int2 w = __ldg(p + chunk_index(c, s, 0, 3, 1));
      L.u[2 * c] = mk(lo16(w.x) * kInvFix, hi16(w.x) * kInvFix);
      L.u[2 * c + 1] = mk(lo16(w.y) * kInvFix, hi16(w.y) * kInvFix);
    }
    su3_reconstruct(L);
  }
  template <class RS>
  static QCU_D void store(void* gauge, int Vh_pad, int mu, int parity, int s, const Link<RS>& L) {
    int2* p = static_cast<int2*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 3;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int2 w;
      w.x = pack16((float)L.u[2 * c].re * kFix, (float)L.u[2 * c].im * kFix);
      w.y = pack16((float)L.u[2 * c + 1].re * kFix, (float)L.u[2 * c + 1].im * kFix);
      p[chunk_index(c, s, 0, 3, 1)] = w;
    }
  }
};

// All 18 reals in FP32: 5 chunks of float4 (the last half used). Nothing to
// decode or rebuild; 80 bytes per link, shared by every RHS lane of a site.
template <> struct LinkIO<LINK_SINGLE18> {
  typedef float R;
  static QCU_D void load(Link<R>& L, const void* gauge, int Vh_pad, int mu, int parity, int s) {
    const float4* p = static_cast<const float4*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 5;
    float4 w[5];
#pragma unroll
    for (int c = 0; c < 5; c++) w[c] = __ldg(p + chunk_index(c, s, 0, 5, 1));
#pragma unroll
    for (int c = 0; c < 4; c++) {
      L.u[2 * c] = mk(w[c].x, w[c].y);
      L.u[2 * c + 1] = mk(w[c].z, w[c].w);
    }
    L.u[8] = mk(w[4].x, w[4].y);
  }
  // L must hold all nine entries (third row rebuilt)
  template <class RS>
  static QCU_D void store(void* gauge, int Vh_pad, int mu, int parity, int s, const Link<RS>& L) {
    float4* p = static_cast<float4*>(gauge) + (size_t)(mu * 2 + parity) * Vh_pad * 5;
#pragma unroll
    for (int c = 0; c < 4; c++)
      p[chunk_index(c, s, 0, 5, 1)] = make_float4((float)L.u[2 * c].re, (float)L.u[2 * c].im,
                                                  (float)L.u[2 * c + 1].re, (float)L.u[2 * c + 1].im);
    p[chunk_index(4, s, 0, 5, 1)] = make_float4((float)L.u[8].re, (float)L.u[8].im, 0.f, 0.f);
  }
};

// ---------------- packed clover ----------------
// One Hermitian 6x6 block: d[6] real diagonal, o[15] strictly-lower entries
// (row i > column j at tri_index(i,j)).
template <class R> struct HermBlock {
  R d[6];
  Cplx<R> o[15];
};

// v <- B v for one block
template <class R> QCU_D void herm_apply(const HermBlock<R>& B, Cplx<R> v[6]) {
  Cplx<R> o[6];
#pragma unroll
  for (int i = 0; i < 6; i++) o[i] = B.d[i] * v[i];
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++) {
      cmac(o[i], B.o[tri_index(i, j)], v[j]);
      cmac_conj(o[j], B.o[tri_index(i, j)], v[i]);
    }
#pragma unroll
  for (int i = 0; i < 6; i++) v[i] = o[i];
}

template <int P> struct CloverIO;

// clover field: [parity] sub-arrays of Vh_pad sites each; clover_index picks a
// whole field (several kappa*c_sw values can be resident side by side).
template <> struct CloverIO<PREC_DOUBLE> {
  typedef double R;
  static QCU_D void load_block(HermBlock<R>& B, const void* clov, int Vh_pad, int parity, int s, int b) {
    const double2* p = static_cast<const double2*>(clov) + (size_t)parity * Vh_pad * 36;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      double2 w = __ldg(p + chunk_index(b * 18 + k, s, 0, 36, 1));
      B.d[2 * k] = w.x;
      B.d[2 * k + 1] = w.y;
    }
#pragma unroll
    for (int k = 0; k < 15; k++) {
      double2 w = __ldg(p + chunk_index(b * 18 + 3 + k, s, 0, 36, 1));
      B.o[k] = mk(w.x, w.y);
    }
  }
  template <class RS>
  static QCU_D void store_block(void* clov, int Vh_pad, int parity, int s, int b, const HermBlock<RS>& B, float*) {
    double2* p = static_cast<double2*>(clov) + (size_t)parity * Vh_pad * 36;
#pragma unroll
    for (int k = 0; k < 3; k++) p[chunk_index(b * 18 + k, s, 0, 36, 1)] = make_double2(B.d[2 * k], B.d[2 * k + 1]);
#pragma unroll
    for (int k = 0; k < 15; k++) p[chunk_index(b * 18 + 3 + k, s, 0, 36, 1)] = make_double2(B.o[k].re, B.o[k].im);
  }
};

// single: the two blocks interleaved element by element, so that one 16-byte
// chunk holds the same two elements of both blocks: element e of block b
// (e = 0..35 in the order d0..d5, o0.re, o0.im, ..., o14.re, o14.im) is float
// 2e+b of the site's 72, i.e. chunk q = (b0[2q], b1[2q], b0[2q+1], b1[2q+1]).
// clover_apply_packed multiplies both blocks at once with paired FP32
// instructions, lane 0 = block 0, lane 1 = block 1.
template <> struct CloverIO<PREC_SINGLE> {
  typedef float R;
  template <class RS>
  static QCU_D void store_block(void* clov, int Vh_pad, int parity, int s, int b, const HermBlock<RS>& B, float*) {
    float4* p = static_cast<float4*>(clov) + (size_t)parity * Vh_pad * 18;
    float a[36];
#pragma unroll
    for (int k = 0; k < 6; k++) a[k] = (float)B.d[k];
#pragma unroll
    for (int k = 0; k < 15; k++) { a[6 + 2 * k] = (float)B.o[k].re; a[7 + 2 * k] = (float)B.o[k].im; }
#pragma unroll
    for (int q = 0; q < 18; q++) {
      float* c = reinterpret_cast<float*>(p + chunk_index(q, s, 0, 18, 1));
      c[b] = a[2 * q];
      c[2 + b] = a[2 * q + 1];
    }
  }
};

template <> struct CloverIO<PREC_HALF> {
  typedef float R;
  // 72 int16 per site = 9 int4 chunks; the norm array ([parity][Vh_pad] floats)
  // follows the chunk array of both parities.
  static QCU_D const float* norms(const void* clov, int Vh_pad) {
    return reinterpret_cast<const float*>(static_cast<const int4*>(clov) + (size_t)2 * Vh_pad * 9);
  }
  static QCU_D int word(const int4* w, int k) {
    const int4 c = w[k >> 2];
    int l = k & 3;
    return l == 0 ? c.x : (l == 1 ? c.y : (l == 2 ? c.z : c.w));
  }
  static QCU_D void decode(HermBlock<R>& B, const int4 w[9], int b, float nm) {
    float a[36];
#pragma unroll
    for (int k = 0; k < 18; k++) {
      int v = word(w, b * 18 + k);
      a[2 * k] = lo16(v) * nm;
      a[2 * k + 1] = hi16(v) * nm;
    }
#pragma unroll
    for (int k = 0; k < 6; k++) B.d[k] = a[k];
#pragma unroll
    for (int k = 0; k < 15; k++) B.o[k] = mk(a[6 + 2 * k], a[7 + 2 * k]);
  }
  static QCU_D void load_block(HermBlock<R>& B, const void* clov, int Vh_pad, int parity, int s, int b) {
    const int4* p = static_cast<const int4*>(clov) + (size_t)parity * Vh_pad * 9;
    int4 w[9];
#pragma unroll
    for (int c = 0; c < 9; c++) w[c] = __ldg(p + chunk_index(c, s, 0, 9, 1));
    float nm = __ldg(norms(clov, Vh_pad) + (size_t)parity * Vh_pad + s) * kInvFix;
    decode(B, w, b, nm);
  }
  // stores both blocks; the site norm is the largest |real| over both
  template <class RS>
  static QCU_D void store_site(void* clov, int Vh_pad, int parity, int s, const HermBlock<RS> B[2]) {
    float mx = 0.f;
#pragma unroll
    for (int b = 0; b < 2; b++) {
#pragma unroll
      for (int k = 0; k < 6; k++) mx = fmaxf(mx, fabsf((float)B[b].d[k]));
#pragma unroll
      for (int k = 0; k < 15; k++) mx = fmaxf(mx, fmaxf(fabsf((float)B[b].o[k].re), fabsf((float)B[b].o[k].im)));
    }
    float sc = mx > 0.f ? kFix / mx : 0.f;
    int words[36];
#pragma unroll
    for (int b = 0; b < 2; b++) {
#pragma unroll
      for (int k = 0; k < 3; k++) words[b * 18 + k] = pack16((float)B[b].d[2 * k] * sc, (float)B[b].d[2 * k + 1] * sc);
#pragma unroll
      for (int k = 0; k < 15; k++) words[b * 18 + 3 + k] = pack16((float)B[b].o[k].re * sc, (float)B[b].o[k].im * sc);
    }
    int4* p = static_cast<int4*>(clov) + (size_t)parity * Vh_pad * 9;
#pragma unroll
    for (int c = 0; c < 9; c++) p[chunk_index(c, s, 0, 9, 1)] = make_int4(words[4 * c], words[4 * c + 1], words[4 * c + 2], words[4 * c + 3]);
    float* nrm = const_cast<float*>(norms(clov, Vh_pad));
    nrm[(size_t)parity * Vh_pad + s] = mx;
  }
};

// v <- blockdiag(B0, B1) v with the single-precision clover, both blocks in
// the two lanes of paired FP32 instructions (sm_100 FFMA2/FMUL2): per site
// 12 paired multiplies and 120 paired FMAs instead of twice as many scalar ones.
QCU_D void clover_apply_packed(Spinor<float>& v, const void* clov, int Vh_pad, int parity, int s) {
  const float4* p = static_cast<const float4*>(clov) + (size_t)parity * Vh_pad * 18;
  float2 D[6], Mre[15], Mim[15];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const float4 w = __ldg(p + chunk_index(q, s, 0, 18, 1));
    D[2 * q] = make_float2(w.x, w.y);
    D[2 * q + 1] = make_float2(w.z, w.w);
  }
#pragma unroll
  for (int k = 0; k < 15; k++) {
    const float4 w = __ldg(p + chunk_index(3 + k, s, 0, 18, 1));
    Mre[k] = make_float2(w.x, w.y);
    Mim[k] = make_float2(w.z, w.w);
  }
  float2 Vre[6], Vim[6], Ore[6], Oim[6];
#pragma unroll
  for (int j = 0; j < 6; j++) {
    Vre[j] = make_float2(v.c[j].re, v.c[6 + j].re);
    Vim[j] = make_float2(v.c[j].im, v.c[6 + j].im);
    Ore[j] = fmul2(D[j], Vre[j]);
    Oim[j] = fmul2(D[j], Vim[j]);
  }
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++) {
      const int k = tri_index(i, j);
      // o_i += M_ij v_j
      Ore[i] = ffma2(Mre[k], Vre[j], Ore[i]);
      Ore[i] = ffma2(fneg2(Mim[k]), Vim[j], Ore[i]);
      Oim[i] = ffma2(Mre[k], Vim[j], Oim[i]);
      Oim[i] = ffma2(Mim[k], Vre[j], Oim[i]);
      // o_j += conj(M_ij) v_i
      Ore[j] = ffma2(Mre[k], Vre[i], Ore[j]);
      Ore[j] = ffma2(Mim[k], Vim[i], Ore[j]);
      Oim[j] = ffma2(Mre[k], Vim[i], Oim[j]);
      Oim[j] = ffma2(fneg2(Mim[k]), Vre[i], Oim[j]);
    }
#pragma unroll
  for (int j = 0; j < 6; j++) {
    v.c[j] = mk(Ore[j].x, Oim[j].x);
    v.c[6 + j] = mk(Ore[j].y, Oim[j].y);
  }
}

// v <- blockdiag(B0, B1) v with the site's packed clover (one block at a time
// for double; the 16-bit form is fetched in one go, 9 x 16 bytes).
// The same with scalar FP32 instructions, one block after the other.
QCU_D void clover_apply_single_scalar(Spinor<float>& v, const void* clov, int Vh_pad, int parity, int s) {
  const float4* p = static_cast<const float4*>(clov) + (size_t)parity * Vh_pad * 18;
  float4 w[18];
#pragma unroll
  for (int q = 0; q < 18; q++) w[q] = __ldg(p + chunk_index(q, s, 0, 18, 1));
#pragma unroll
  for (int b = 0; b < 2; b++) {
    HermBlock<float> B;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      B.d[2 * q] = b ? w[q].y : w[q].x;
      B.d[2 * q + 1] = b ? w[q].w : w[q].z;
    }
#pragma unroll
    for (int k = 0; k < 15; k++) B.o[k] = b ? mk(w[3 + k].y, w[3 + k].w) : mk(w[3 + k].x, w[3 + k].z);
    Cplx<float> t[6];
#pragma unroll
    for (int i = 0; i < 6; i++) t[i] = v.c[6 * b + i];
    herm_apply(B, t);
#pragma unroll
    for (int i = 0; i < 6; i++) v.c[6 * b + i] = t[i];
  }
}

// Paired (1) or scalar (0) FP32 clover multiply. Measured on B200 at 32^4 in
// the fused CG stencil: no gain from pairing (117 vs 120 us at 1 RHS, 1349 vs
// 1369 us at 16 RHS), so the scalar form is the default.
#ifndef QCU_CLOVER_FFMA2
#define QCU_CLOVER_FFMA2 0
#endif

template <int P, class R>
QCU_D void clover_apply_site(Spinor<R>& v, const void* clov, int Vh_pad, int parity, int s) {
  if constexpr (P == PREC_SINGLE) {
    static_assert(sizeof(R) == sizeof(float), "the single-precision clover is applied in FP32");
#if QCU_CLOVER_FFMA2
    clover_apply_packed(v, clov, Vh_pad, parity, s);
#else
    clover_apply_single_scalar(v, clov, Vh_pad, parity, s);
#endif
  } else if constexpr (P == PREC_HALF) {
    const int4* p = static_cast<const int4*>(clov) + (size_t)parity * Vh_pad * 9;
    int4 w[9];
#pragma unroll
    for (int c = 0; c < 9; c++) w[c] = __ldg(p + chunk_index(c, s, 0, 9, 1));
    float nm = __ldg(CloverIO<PREC_HALF>::norms(clov, Vh_pad) + (size_t)parity * Vh_pad + s) * kInvFix;
#pragma unroll
    for (int b = 0; b < 2; b++) {
      HermBlock<float> B;
      CloverIO<PREC_HALF>::decode(B, w, b, nm);
      Cplx<float> t[6];
#pragma unroll
      for (int i = 0; i < 6; i++) t[i] = mk((float)v.c[6 * b + i].re, (float)v.c[6 * b + i].im);
      herm_apply(B, t);
#pragma unroll
      for (int i = 0; i < 6; i++) v.c[6 * b + i] = mk((R)t[i].re, (R)t[i].im);
    }
  } else {
#pragma unroll
    for (int b = 0; b < 2; b++) {
      HermBlock<typename CloverIO<P>::R> B;
      CloverIO<P>::load_block(B, clov, Vh_pad, parity, s, b);
      Cplx<typename CloverIO<P>::R> t[6];
#pragma unroll
      for (int i = 0; i < 6; i++) t[i] = mk((typename CloverIO<P>::R)v.c[6 * b + i].re, (typename CloverIO<P>::R)v.c[6 * b + i].im);
      herm_apply(B, t);
#pragma unroll
      for (int i = 0; i < 6; i++) v.c[6 * b + i] = mk((R)t[i].re, (R)t[i].im);
    }
  }
}

// bytes of a clover field (both parities) in the given precision
inline size_t clover_field_bytes(int P, int Vh_pad) {
  if (P == PREC_DOUBLE) return (size_t)2 * Vh_pad * 36 * 16;
  if (P == PREC_SINGLE) return (size_t)2 * Vh_pad * 18 * 16;
  return (size_t)2 * Vh_pad * 9 * 16 + (size_t)2 * Vh_pad * 4;
}
inline size_t gauge_field_bytes(int P, int Vh_pad) {
  if (P == LINK_SINGLE18) return (size_t)8 * Vh_pad * 5 * 16;
  if (P == PREC_DOUBLE) return (size_t)8 * Vh_pad * 6 * 16;
  if (P == PREC_SINGLE) return (size_t)8 * Vh_pad * 3 * 16;
  return (size_t)8 * Vh_pad * 3 * 8;
}
inline size_t spinor_field_bytes(int P, int Vh_pad, int nrhs) {
  if (P == PREC_DOUBLE) return (size_t)Vh_pad * nrhs * 12 * 16;
  if (P == PREC_SINGLE) return (size_t)Vh_pad * nrhs * 6 * 16;
  return (size_t)Vh_pad * nrhs * 3 * 16;
}
inline size_t spinor_norm_bytes(int P, int Vh_pad, int nrhs) {
  return P == PREC_HALF ? (size_t)Vh_pad * nrhs * 4 : 0;
}

}  // namespace qcu
