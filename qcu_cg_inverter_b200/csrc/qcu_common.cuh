// Common device/host definitions for the B200 Wilson-clover solver.
//
// Conventions (they follow the reference library, YellowBicycleee/Qcu_Cg_Inverter,
// paths below are inside its cg_inverter/ directory):
//  * even-odd checkerboard: parity p holds sites with (x+y+z+t)&1 == p; the
//    checkerboard index is s = ((t*Lz + z)*Ly + y)*(Lx/2) + x/2 and the full x
//    coordinate is x = 2*(x/2) + ((y+z+t+p)&1) (include/qcu_point.cuh:20-72);
//  * spinor component k = spin*3 + colour, DeGrand-Rossi gamma basis as written
//    out in the hopping kernel (src/qcu_clover_dslash.cu:570-772);
//  * links keep their first two rows; the third is conj(row0 x row1)
//    (src/qcu_clover_dslash.cu:11-16);
//  * the clover matrix of a site is two 6x6 Hermitian blocks acting on spins
//    {0,1} and {2,3} (src/qcu_clover_dslash.cu:461-506).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <cuda_fp16.h>

#define QCU_HD __host__ __device__ __forceinline__
#define QCU_D __device__ __forceinline__

namespace qcu {

// ---------------------------------------------------------------------------
// complex arithmetic
// ---------------------------------------------------------------------------
template <class R> struct Cplx {
  R re, im;
};
template <class R> QCU_HD Cplx<R> mk(R a, R b) { return Cplx<R>{a, b}; }
template <class R> QCU_HD Cplx<R> operator+(Cplx<R> a, Cplx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <class R> QCU_HD Cplx<R> operator-(Cplx<R> a, Cplx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <class R> QCU_HD Cplx<R> operator*(Cplx<R> a, Cplx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class R> QCU_HD Cplx<R> operator*(R s, Cplx<R> a) { return {s * a.re, s * a.im}; }
template <class R> QCU_HD Cplx<R> conj(Cplx<R> a) { return {a.re, -a.im}; }
template <class R> QCU_HD Cplx<R> mul_i(Cplx<R> a) { return {-a.im, a.re}; }  // i*a
template <class R> QCU_HD Cplx<R>& operator+=(Cplx<R>& a, Cplx<R> b) { a.re += b.re; a.im += b.im; return a; }
template <class R> QCU_HD Cplx<R>& operator-=(Cplx<R>& a, Cplx<R> b) { a.re -= b.re; a.im -= b.im; return a; }
// a += b*c, as four fused multiply-adds into the accumulator (written as
// a + (x - y) the compiler may not reassociate, and emits a multiply, an FMA
// and an add per component)
template <class R> QCU_HD void cmac(Cplx<R>& a, Cplx<R> b, Cplx<R> c) {
  a.re = fma(b.re, c.re, a.re);
  a.re = fma(-b.im, c.im, a.re);
  a.im = fma(b.re, c.im, a.im);
  a.im = fma(b.im, c.re, a.im);
}
// a += conj(b)*c
template <class R> QCU_HD void cmac_conj(Cplx<R>& a, Cplx<R> b, Cplx<R> c) {
  a.re = fma(b.re, c.re, a.re);
  a.re = fma(b.im, c.im, a.re);
  a.im = fma(b.re, c.im, a.im);
  a.im = fma(-b.im, c.re, a.im);
}

template <class R> struct Spinor {
  Cplx<R> c[12];  // spin*3 + colour
};
template <class R> struct Link {
  Cplx<R> u[9];   // row-major 3x3
};

template <class R> QCU_HD void su3_reconstruct(Link<R>& L) {
  // row 3 = conj(row1 x row2)
  L.u[6] = conj(L.u[1] * L.u[5] - L.u[2] * L.u[4]);
  L.u[7] = conj(L.u[2] * L.u[3] - L.u[0] * L.u[5]);
  L.u[8] = conj(L.u[0] * L.u[4] - L.u[1] * L.u[3]);
}

// ---------------------------------------------------------------------------
// lattice geometry
// ---------------------------------------------------------------------------
// Division by a lattice extent d without a division instruction (Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994):
// with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (umulhi(m, n) + n) >> l for every 0 <= n < 2^31.
struct FastDiv {
  unsigned m;
  int l, d;
};
inline FastDiv make_fastdiv(int d) {
  FastDiv f;
  int l = 0;
  while ((1ll << l) < d) l++;
  f.l = l;
  f.d = d;
  f.m = (unsigned)((((unsigned long long)1 << 32) * (((unsigned long long)1 << l) - (unsigned long long)d)) /
                       (unsigned long long)d + 1);
  return f;
}
QCU_HD int fdiv(int n, const FastDiv& f) {
#ifdef __CUDA_ARCH__
  return (int)((__umulhi(f.m, (unsigned)n) + (unsigned)n) >> f.l);
#else
  return n / f.d;
#endif
}

struct Geom {
  int Lx, Ly, Lz, Lt;
  int Lxh;      // Lx/2
  int Vh;       // sites per parity
  int Vh_pad;   // sites per parity block of every field: Vh rounded up to the 32-site block, plus the ghost slices
  int sy, sz, st;  // checkerboard strides of y, z, t: Lxh, Lxh*Ly, Lxh*Ly*Lz
  FastDiv dxh, dy, dz;  // division by Lxh, Ly, Lz
  // t-slab of a lattice decomposed along t (tdd = 1): the hops across the
  // slab's t faces read ghost slices appended to every parity block, the
  // forward one at sites [gfwd, gfwd + st), the backward one at [gbwd, gbwd +
  // st), filled by the halo exchange; tdd = 0: periodic wrap inside the lattice
  int tdd, gfwd, gbwd;
  // which t faces are the lattice's boundary, where hops take the factor bc_t:
  // bit 0 the backward face (t = 0), bit 1 the forward one (t = Lt - 1)
  int tbc;
};

inline Geom make_geom(const int L[4]) {
  Geom g;
  g.Lx = L[0]; g.Ly = L[1]; g.Lz = L[2]; g.Lt = L[3];
  g.Lxh = L[0] / 2;
  g.Vh = g.Lxh * g.Ly * g.Lz * g.Lt;
  g.Vh_pad = (g.Vh + 31) & ~31;
  g.sy = g.Lxh;
  g.sz = g.Lxh * g.Ly;
  g.st = g.Lxh * g.Ly * g.Lz;
  g.dxh = make_fastdiv(g.Lxh);
  g.dy = make_fastdiv(g.Ly);
  g.dz = make_fastdiv(g.Lz);
  g.tdd = 0;
  g.gfwd = g.gbwd = 0;
  g.tbc = 3;
  return g;
}

// The slab of rank `rank` of `nranks` of a lattice decomposed along t: local
// time extent L[3] / nranks (even, so that local and global parity agree),
// ghost slices after the slab's sites. Needs the slice (Lxh*Ly*Lz sites) to be
// a whole number of 32-site blocks, so that a slice is a contiguous range of
// every field; slab_ok() checks that.
inline bool slab_ok(const int L[4], int nranks) {
  if (nranks < 1 || L[3] % nranks) return false;
  const int lt = L[3] / nranks;
  return lt >= 2 && lt % 2 == 0 && ((L[0] / 2) * L[1] * L[2]) % 32 == 0;
}
inline Geom make_geom_slab(const int L[4], int nranks, int rank) {
  const int Ll[4] = {L[0], L[1], L[2], L[3] / nranks};
  Geom g = make_geom(Ll);
  g.tdd = 1;
  g.gfwd = g.Vh;  // a multiple of 32 (slab_ok)
  g.gbwd = g.Vh + g.st;
  g.Vh_pad = g.Vh + 2 * g.st;
  g.tbc = (rank == 0 ? 1 : 0) | (rank == nranks - 1 ? 2 : 0);
  return g;
}

// Coordinates and the 8 neighbours of a checkerboard site. The x step follows
// Point::move (include/qcu_point.cuh:26-36): with eo = (y+z+t)&1 the forward
// x neighbour has x/2+1 when eo != parity (else the same x/2), the backward
// one x/2-1 when eo == parity; every direction wraps periodically.
struct Nbrs {
  int fwd[4], bwd[4];
  int t;       // time coordinate
  bool tf, tb;  // the forward / backward t hop crosses the lattice's boundary (takes bc_t)
};

QCU_HD Nbrs neighbours(const Geom& g, int s, int parity) {
  Nbrs n;
  int r = fdiv(s, g.dxh);
  const int xh = s - r * g.Lxh;
  const int r2 = fdiv(r, g.dy);
  const int y = r - r2 * g.Ly;
  const int t = fdiv(r2, g.dz);
  const int z = r2 - t * g.Lz;
  n.t = t;
  int eo = (y + z + t) & 1;
  int xf = (eo != parity) ? (xh + 1 == g.Lxh ? 0 : xh + 1) : xh;
  int xb = (eo == parity) ? (xh == 0 ? g.Lxh - 1 : xh - 1) : xh;
  n.fwd[0] = s - xh + xf;
  n.bwd[0] = s - xh + xb;
  n.fwd[1] = (y + 1 == g.Ly) ? s - (g.Ly - 1) * g.sy : s + g.sy;
  n.bwd[1] = (y == 0) ? s + (g.Ly - 1) * g.sy : s - g.sy;
  n.fwd[2] = (z + 1 == g.Lz) ? s - (g.Lz - 1) * g.sz : s + g.sz;
  n.bwd[2] = (z == 0) ? s + (g.Lz - 1) * g.sz : s - g.sz;
  const bool top = t + 1 == g.Lt, bot = t == 0;
  n.tf = top && (g.tbc & 2);
  n.tb = bot && (g.tbc & 1);
  if (g.tdd) {  // across the slab's faces: the ghost slices
    n.fwd[3] = top ? g.gfwd + (s - (g.Lt - 1) * g.st) : s + g.st;
    n.bwd[3] = bot ? g.gbwd + s : s - g.st;
  } else {
    n.fwd[3] = top ? s - (g.Lt - 1) * g.st : s + g.st;
    n.bwd[3] = bot ? s + (g.Lt - 1) * g.st : s - g.st;
  }
  return n;
}

// ---------------------------------------------------------------------------
// internal field layout: site-blocked, vectorised SoA
// ---------------------------------------------------------------------------
// Every field is a sequence of 16-byte chunks. Sites are grouped in blocks of
// 32 (one warp); within a block, chunk c of all 32 sites (and, for batched
// fields, of all nrhs right-hand sides of each site) is contiguous:
//     chunk(c, s, r) = ((s/32 * NC + c) * 32 + s%32) * nrhs + r
// so a warp reading chunk c of 32 consecutive sites reads 512*nrhs contiguous
// bytes, and all chunks of a site block sit within a few KB.
//
// Kernels compute the index in 32-bit unsigned arithmetic (the pointer add
// then takes one wide multiply-add), so a field holds fewer than 2^32 chunks
// per parity block: field_index32_ok is checked wherever fields are sized.
QCU_HD size_t chunk_index(int c, int s, int r, int NC, int nrhs) {
#ifdef __CUDA_ARCH__
  return (((((unsigned)s >> 5) * (unsigned)NC + (unsigned)c) << 5) + ((unsigned)s & 31u)) * (unsigned)nrhs + (unsigned)r;
#else
  return ((size_t)((s >> 5) * NC + c) * 32 + (s & 31)) * (size_t)nrhs + r;
#endif
}
// per-site, per-RHS scalars (16-bit spinor norms)
QCU_HD size_t site_rhs_index(int s, int r, int nrhs) {
#ifdef __CUDA_ARCH__
  return (unsigned)s * (unsigned)nrhs + (unsigned)r;
#else
  return (size_t)s * nrhs + r;
#endif
}
// the largest chunk count per site of any field (FP64 clover: 36; FP64
// spinors: 12 per RHS)
inline bool field_index32_ok(long long Vh_pad, long long nrhs) {
  const long long per_site = 12 * nrhs > 36 ? 12 * nrhs : 36;
  return Vh_pad > 0 && nrhs > 0 && Vh_pad * per_site < (1LL << 32);
}

// ---------------------------------------------------------------------------
// precision traits
// ---------------------------------------------------------------------------
enum Prec : int { PREC_DOUBLE = 0, PREC_SINGLE = 1, PREC_HALF = 2 };

// Link storage formats (LinkIO): the three above keep 12 reals (two rows) and
// rebuild the third row; LINK_SINGLE18 keeps all 18 reals in FP32 (80 bytes
// with padding), so a kernel does no decoding and no reconstruction.
// LINK_HALF_RAW is the 16-bit 12-real storage of PREC_HALF read by the
// single-RHS compact kernels: entries stay in units of the 16-bit grid
// (x 32767) and the stencil folds the 1/32767 into its per-neighbour scale.
enum LinkFormat : int { LINK_SINGLE18 = 3, LINK_HALF_RAW = 4 };

// Operator variants (the `prec` argument of launch_dslash): spinor, link and
// clover storage of one stencil instantiation.
enum OpVariant : int {
  OP_DOUBLE = 0,     // FP64 spinors, FP64 12-real links, FP64 clover
  OP_SINGLE = 1,     // FP32 spinors, FP32 12-real links, FP32 clover
  OP_HALF = 2,       // 16-bit spinors, 16-bit 12-real links, 16-bit clover
  OP_HALF_FAST = 3,  // 16-bit spinors, FP32 18-real links, FP32 clover
  // the same storage as OP_HALF_FAST; the kernels its launches use for a
  // single RHS (block-paired epilogues at 128 registers)
  OP_HALF_FAST_1 = 4,
  // the same storage again; the kernels of its batched launches: two
  // right-hand sides per thread in the lanes of paired FP32 instructions
  OP_HALF_FAST_2 = 5,
  // the storage of OP_DOUBLE; the kernels of its batched launches (a register
  // cap and row-at-a-time reconstruction)
  OP_DOUBLE_BATCH = 6,
  // the storage of OP_HALF (everything 16-bit); the kernels its single-RHS
  // launches use (paired decode, block-paired epilogues)
  OP_HALF_1 = 7,
  // the kernels of OP_HALF_FAST_2 with the t neighbours' words (8), or the z
  // and t neighbours' (9), staged in shared memory
  OP_HALF_FAST_2T = 8,
  OP_HALF_FAST_2Z = 9,
};
// staged directions of an RHS-paired kernel family
__host__ __device__ constexpr int op_staged(int op) {
  return op == OP_HALF_FAST_2T ? 1 : op == OP_HALF_FAST_2Z ? 2 : 0;
}
__host__ __device__ constexpr bool op_pair(int op) { return op == OP_HALF_FAST_2 || op_staged(op) > 0; }
// Storage of the sloppy solver's accumulators (the partial solution x_lo and
// the iterated residual r) for a sloppy spinor precision: FP64 for FP64, FP32
// for FP32, and for 16-bit solves 16-bit like their other spinors (QCU_ACC16
// 1) or FP32 (0). Measured with 16-bit accumulators: the same iteration and
// reliable-update counts (16^3x32: 50 and 6; 48-RHS 24^3x48: 47-50), the CG
// update stencil 666 -> 587 us (24^3x48, 16 RHS), the 48-RHS batch 0.512 ->
// 0.494 s, config 2 3.50 -> 3.43 ms. The reliable updates bound the error the
// 16-bit recurrences add.
#ifndef QCU_ACC16
#define QCU_ACC16 1
#endif
__host__ __device__ constexpr int acc_prec(int ps) {
  return ps == PREC_DOUBLE ? (int)PREC_DOUBLE : (ps == PREC_HALF && QCU_ACC16) ? (int)PREC_HALF : (int)PREC_SINGLE;
}
__host__ __device__ constexpr bool op_fast(int op) {
  return op == OP_HALF_FAST || op == OP_HALF_FAST_1 || op_pair(op);
}
__host__ __device__ constexpr int op_base(int op) {
  return op == OP_DOUBLE_BATCH ? (int)OP_DOUBLE : op == OP_HALF_1 ? (int)OP_HALF : op;
}
__host__ __device__ constexpr int op_spinor_prec(int op) { return op_fast(op) ? (int)PREC_HALF : op_base(op); }
__host__ __device__ constexpr int op_link_format(int op) { return op_fast(op) ? (int)LINK_SINGLE18 : op_base(op); }
__host__ __device__ constexpr int op_clover_prec(int op) { return op_fast(op) ? (int)PREC_SINGLE : op_base(op); }

// 16-bit storage is fixed point: a real v in [-1,1] is stored as
// round(v*32767); spinors and clover blocks carry one float norm per site so
// that their largest component maps to 1.
constexpr float kFix = 32767.0f;
constexpr float kInvFix = 1.0f / 32767.0f;

// spinor chunks per site: 12 complex in 16 bytes
template <int P> struct SpinorChunks;
template <> struct SpinorChunks<PREC_DOUBLE> { static constexpr int NC = 12; };  // double2
template <> struct SpinorChunks<PREC_SINGLE> { static constexpr int NC = 6; };   // float4
template <> struct SpinorChunks<PREC_HALF> { static constexpr int NC = 3; };     // 8 x int16
// gauge: 12 reals per link
template <int P> struct GaugeChunks;
template <> struct GaugeChunks<PREC_DOUBLE> { static constexpr int NC = 6; };   // double2
template <> struct GaugeChunks<PREC_SINGLE> { static constexpr int NC = 3; };   // float4
template <> struct GaugeChunks<PREC_HALF> { static constexpr int NC = 3; };     // 4 x int16 (8 bytes)
// packed clover: 72 reals per site (two Hermitian 6x6 blocks, 36 reals each:
// 6 real diagonal entries, then the 15 strictly-lower entries row by row)
template <int P> struct CloverChunks;
template <> struct CloverChunks<PREC_DOUBLE> { static constexpr int NC = 36; };  // double2
template <> struct CloverChunks<PREC_SINGLE> { static constexpr int NC = 18; };  // float4
template <> struct CloverChunks<PREC_HALF> { static constexpr int NC = 9; };     // 8 x int16

template <int P> struct CompReal { typedef float type; };
template <> struct CompReal<PREC_DOUBLE> { typedef double type; };

// bytes per site of each field kind
template <int P> constexpr int spinor_bytes() { return P == PREC_DOUBLE ? 192 : (P == PREC_SINGLE ? 96 : 52); }
template <int P> constexpr int link_bytes() { return P == PREC_DOUBLE ? 96 : (P == PREC_SINGLE ? 48 : 24); }
template <int P> constexpr int clover_bytes() { return P == PREC_DOUBLE ? 576 : (P == PREC_SINGLE ? 288 : 148); }

// off-diagonal packed index of (i,j), i > j, of a 6x6 Hermitian block
QCU_HD int tri_index(int i, int j) { return i * (i - 1) / 2 + j; }

// ---------------------------------------------------------------------------
// counter-based random numbers (SplitMix64 streams keyed by (seed, object))
// ---------------------------------------------------------------------------
QCU_HD uint64_t sm64_next(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
QCU_HD uint64_t stream_init(uint64_t seed, uint64_t object) {
  uint64_t s = seed ^ 0xD1B54A32D192ED03ull;
  s += object * 0x632BE59BD9B4E019ull;
  (void)sm64_next(s);
  return s;
}

}  // namespace qcu
