// Clover term: build A = 1 + csw_eff*T from the four-leaf field strength and
// factor each 6x6 chiral block once in FP64 (root-free Cholesky, A = L D L^H),
// storing A and A^-1 packed (72 reals per site) in the internal layout.
//
// T follows the reference exactly (src/qcu_clover_dslash.cu:173-458, 509-544):
//   Q_munu = F1+F2+F3+F4 (four leaves around x), G = Q - Q^dag,
//   T = (-1/16)*2 * sum_{mu<nu} (spin phase table) (x) G,
// no trace subtraction; csw_eff = 1 reproduces the reference, csw_eff =
// kappa*c_sw gives A = 1 - (kappa c_sw / 2) sigma.F for the physical operator.
// The reference builds 32 shifted copies of the gauge field for the leaves
// (src/qcu_communicator.cu:755-980, 1270-1297, 38.7 GB transient at 32^3x64);
// here each thread indexes the neighbouring links directly.
//
// Kernel shape: a block handles 32 sites; thread (plane, site) computes the
// six G_munu into shared memory, then thread (block b, site) assembles chiral
// block b, factors it and writes A and A^-1.
#include "qcu_cg_state.cuh"
#include "qcu_fields.cuh"
#include "qcu_kernels.cuh"

namespace qcu {

struct CloverBuildArgs {
  Geom g;
  const void* gauge;       // internal FP64 links
  void* T64;               // the kappa-independent field term T/(kappa c_sw), packed FP64 (see below)
  double csw_eff;
  void* A64;               // packed A, FP64 (nullable)
  void* Ainv64;            // packed A^-1, FP64 (nullable)
  void* Ainv32;            // packed A^-1, single (nullable)
  void* Ainv16;            // packed A^-1, 16-bit (nullable)
  int* status;             // [0]: blocks with a non-positive pivot, [1]: blocks with a zero/non-finite pivot
};

// tensorProductAddition spin structure, src/qcu_clover_dslash.cu:210-267: for
// plane pl and row spin sp, the column spin and the phase (re, im).
__constant__ int kPlaneMu[6] = {0, 0, 0, 1, 1, 2};
__constant__ int kPlaneNu[6] = {1, 2, 3, 2, 3, 3};
__constant__ int kColSpin[6][4] = {{0, 1, 2, 3}, {1, 0, 3, 2}, {1, 0, 3, 2}, {1, 0, 3, 2}, {1, 0, 3, 2}, {0, 1, 2, 3}};
__constant__ double kPhRe[6][4] = {{0, 0, 0, 0}, {-1, 1, -1, 1}, {0, 0, 0, 0}, {0, 0, 0, 0}, {-1, 1, 1, -1}, {0, 0, 0, 0}};
__constant__ double kPhIm[6][4] = {{-1, 1, -1, 1}, {0, 0, 0, 0}, {1, 1, -1, -1}, {-1, -1, -1, -1}, {0, 0, 0, 0}, {1, -1, -1, 1}};

typedef Cplx<double> C64;

QCU_D void link_full(Link<double>& U, const Geom& g, const void* gauge, int mu, int x, int y, int z, int t) {
  x = (x + g.Lx) % g.Lx;
  y = (y + g.Ly) % g.Ly;
  z = (z + g.Lz) % g.Lz;
  t = (t + g.Lt) % g.Lt;
  int parity = (x + y + z + t) & 1;
  int s = ((t * g.Lz + z) * g.Ly + y) * g.Lxh + (x >> 1);
  LinkIO<PREC_DOUBLE>::load(U, gauge, g.Vh_pad, mu, parity, s);
}

QCU_D void m_mul(Link<double>& r, const Link<double>& a, const Link<double>& b) {
  Link<double> t;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      C64 acc = a.u[i * 3] * b.u[j];
      cmac(acc, a.u[i * 3 + 1], b.u[3 + j]);
      cmac(acc, a.u[i * 3 + 2], b.u[6 + j]);
      t.u[i * 3 + j] = acc;
    }
  r = t;
}
// r = a * b^dag
QCU_D void m_mul_dag(Link<double>& r, const Link<double>& a, const Link<double>& b) {
  Link<double> t;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      C64 acc = mk(0.0, 0.0);
      cmac(acc, a.u[i * 3], conj(b.u[j * 3]));
      cmac(acc, a.u[i * 3 + 1], conj(b.u[j * 3 + 1]));
      cmac(acc, a.u[i * 3 + 2], conj(b.u[j * 3 + 2]));
      t.u[i * 3 + j] = acc;
    }
  r = t;
}
// r = a^dag * b
QCU_D void m_dag_mul(Link<double>& r, const Link<double>& a, const Link<double>& b) {
  Link<double> t;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      C64 acc = mk(0.0, 0.0);
      cmac_conj(acc, a.u[i], b.u[j]);
      cmac_conj(acc, a.u[3 + i], b.u[3 + j]);
      cmac_conj(acc, a.u[6 + i], b.u[6 + j]);
      t.u[i * 3 + j] = acc;
    }
  r = t;
}

// Q_munu(x): the four leaves of src/qcu_clover_dslash.cu:329-413
//  F1 = U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
//  F2 = U_nu(x) U_mu(x-mu+nu)^dag U_nu(x-mu)^dag U_mu(x-mu)
//  F3 = U_mu(x-mu)^dag U_nu(x-mu-nu)^dag U_mu(x-mu-nu) U_nu(x-nu)
//  F4 = U_nu(x-nu)^dag U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^dag
QCU_D void leaves(Link<double>& Q, const Geom& g, const void* gauge, int x, int y, int z, int t, int mu, int nu) {
  int m[4] = {0, 0, 0, 0}, n[4] = {0, 0, 0, 0};
  m[mu] = 1;
  n[nu] = 1;
  Link<double> a, b, r;
#define LK(U, d, o0, o1, o2, o3) link_full(U, g, gauge, d, x + (o0), y + (o1), z + (o2), t + (o3))
  // F1
  LK(a, mu, 0, 0, 0, 0);
  LK(b, nu, m[0], m[1], m[2], m[3]);
  m_mul(r, a, b);
  LK(b, mu, n[0], n[1], n[2], n[3]);
  m_mul_dag(r, r, b);
  LK(b, nu, 0, 0, 0, 0);
  m_mul_dag(Q, r, b);
  // F2
  LK(a, nu, 0, 0, 0, 0);
  LK(b, mu, n[0] - m[0], n[1] - m[1], n[2] - m[2], n[3] - m[3]);
  m_mul_dag(r, a, b);
  LK(b, nu, -m[0], -m[1], -m[2], -m[3]);
  m_mul_dag(r, r, b);
  LK(b, mu, -m[0], -m[1], -m[2], -m[3]);
  m_mul(r, r, b);
#pragma unroll
  for (int i = 0; i < 9; i++) Q.u[i] += r.u[i];
  // F3
  LK(a, mu, -m[0], -m[1], -m[2], -m[3]);
  LK(b, nu, -m[0] - n[0], -m[1] - n[1], -m[2] - n[2], -m[3] - n[3]);
  // r = a^dag b^dag = (b a)^dag
  m_mul(r, b, a);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = i; j < 3; j++) {
      C64 tij = r.u[i * 3 + j], tji = r.u[j * 3 + i];
      r.u[i * 3 + j] = conj(tji);
      r.u[j * 3 + i] = conj(tij);
    }
  LK(b, mu, -m[0] - n[0], -m[1] - n[1], -m[2] - n[2], -m[3] - n[3]);
  m_mul(r, r, b);
  LK(b, nu, -n[0], -n[1], -n[2], -n[3]);
  m_mul(r, r, b);
#pragma unroll
  for (int i = 0; i < 9; i++) Q.u[i] += r.u[i];
  // F4
  LK(a, nu, -n[0], -n[1], -n[2], -n[3]);
  LK(b, mu, -n[0], -n[1], -n[2], -n[3]);
  m_dag_mul(r, a, b);
  LK(b, nu, m[0] - n[0], m[1] - n[1], m[2] - n[2], m[3] - n[3]);
  m_mul(r, r, b);
  LK(b, mu, 0, 0, 0, 0);
  m_mul_dag(r, r, b);
#pragma unroll
  for (int i = 0; i < 9; i++) Q.u[i] += r.u[i];
#undef LK
}

// Root-free Cholesky A = L D L^H of a packed Hermitian 6x6 block, then
// A^-1 = L^-H D^-1 L^-1 packed the same way. Returns 0 for a positive
// definite block, 1 for a non-positive pivot (the factorisation still holds
// for an indefinite block without a zero leading minor), 2 for a zero or
// non-finite pivot.
QCU_D int ldl_invert(const HermBlock<double>& A, HermBlock<double>& Ai) {
  double D[6];
  C64 L[15];  // strictly lower, tri_index
  int st = 0;
  for (int j = 0; j < 6; j++) {
    double dj = A.d[j];
    for (int k = 0; k < j; k++) {
      C64 l = L[tri_index(j, k)];
      dj -= (l.re * l.re + l.im * l.im) * D[k];
    }
    D[j] = dj;
    if (!(dj > 0.0)) st = st > 1 ? st : 1;
    if (dj == 0.0 || !isfinite(dj)) st = 2;
    double inv = 1.0 / dj;
    for (int i = j + 1; i < 6; i++) {
      C64 acc = A.o[tri_index(i, j)];
      for (int k = 0; k < j; k++) {
        C64 t = L[tri_index(i, k)] * conj(L[tri_index(j, k)]);
        acc -= D[k] * t;
      }
      L[tri_index(i, j)] = inv * acc;
    }
  }
  // X = L^-1 (unit lower triangular): X_ij = -sum_{k=j}^{i-1} L_ik X_kj
  C64 X[15];
  for (int j = 0; j < 6; j++) {
    for (int i = j + 1; i < 6; i++) {
      C64 acc = L[tri_index(i, j)];  // k = j term with X_jj = 1
      for (int k = j + 1; k < i; k++) cmac(acc, L[tri_index(i, k)], X[tri_index(k, j)]);
      X[tri_index(i, j)] = mk(-acc.re, -acc.im);
    }
  }
  // (A^-1)_ij = sum_{k >= i} conj(X_ki) X_kj / D_k, i >= j
  for (int i = 0; i < 6; i++) {
    for (int j = 0; j <= i; j++) {
      C64 acc = mk(0.0, 0.0);
      for (int k = i; k < 6; k++) {
        C64 xki = (k == i) ? mk(1.0, 0.0) : X[tri_index(k, i)];
        C64 xkj = (k == j) ? mk(1.0, 0.0) : X[tri_index(k, j)];
        C64 t = conj(xki) * xkj;
        acc += (1.0 / D[k]) * t;
      }
      if (i == j) Ai.d[i] = acc.re;
      else Ai.o[tri_index(i, j)] = acc;
    }
  }
  return st;
}

// The clover term is A = 1 + csw_eff F, with F the kappa-independent field
// term of the leaves (T at csw_eff = 1). F depends on the gauge field alone,
// so it is built once per field (clover_field_kernel, the four-leaf sums) and
// every clover for a new kappa*c_sw only assembles A from it and factors it
// (clover_assemble_kernel). Measured on B200 with the serving stream, where
// nearly every request brings its own kappa: 334.1-334.5 -> 335.2-335.3 RHS
// solves/s, p99 1.05-1.09 -> 0.91-0.97 s.
__global__ void __launch_bounds__(192) clover_field_kernel(const CloverBuildArgs a) {
  // G_munu for 32 sites: anti-Hermitian 3x3 kept as the full 9 complex
  __shared__ C64 sG[32][6][9];
  const int lane = threadIdx.x;   // site within block
  const int pl = threadIdx.y;     // 0..5
  const int site = blockIdx.x * 32 + lane;  // over both parities: [0, 2*Vh)
  const Geom& g = a.g;
  const int parity = site >= g.Vh ? 1 : 0;
  const int s = site - parity * g.Vh;
  const bool valid = site < 2 * g.Vh;
  if (valid) {
    int xh = s % g.Lxh, rr = s / g.Lxh;
    int y = rr % g.Ly;
    rr /= g.Ly;
    int z = rr % g.Lz, t = rr / g.Lz;
    int x = 2 * xh + ((y + z + t + parity) & 1);
    Link<double> Q;
    leaves(Q, g, a.gauge, x, y, z, t, kPlaneMu[pl], kPlaneNu[pl]);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) sG[lane][pl][i * 3 + j] = Q.u[i * 3 + j] - conj(Q.u[j * 3 + i]);
  }
  __syncthreads();
  if (pl >= 2 || !valid) return;
  const int b = pl;  // chiral block: spins {2b, 2b+1}
  // F for block b (full 6x6 in local memory, then packed as a Hermitian block)
  C64 T[36];
  for (int i = 0; i < 36; i++) T[i] = mk(0.0, 0.0);
  const double coef = -1.0 / 16.0 * 2.0;
  for (int p = 0; p < 6; p++) {
    for (int sl = 0; sl < 2; sl++) {
      int sp = 2 * b + sl;
      int r0 = sl * 3, c0 = (kColSpin[p][sp] & 1) * 3;
      C64 ph = mk(kPhRe[p][sp] * coef, kPhIm[p][sp] * coef);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) T[(r0 + i) * 6 + c0 + j] += ph * sG[lane][p][i * 3 + j];
    }
  }
  HermBlock<double> F;
  for (int i = 0; i < 6; i++) F.d[i] = T[i * 7].re;
  for (int i = 1; i < 6; i++)
    for (int j = 0; j < i; j++) F.o[tri_index(i, j)] = T[i * 6 + j];
  CloverIO<PREC_DOUBLE>::store_block(a.T64, g.Vh_pad, parity, s, b, F, nullptr);
}

// A = 1 + csw_eff F for one chiral block per thread, its LDL^H inverse, and
// the stores of A and A^-1
__global__ void __launch_bounds__(128) clover_assemble_kernel(const CloverBuildArgs a) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // (site over both parities, block)
  const Geom& g = a.g;
  if (idx >= 4 * g.Vh) return;
  const int site = idx >> 1, b = idx & 1;
  const int parity = site >= g.Vh ? 1 : 0;
  const int s = site - parity * g.Vh;
  HermBlock<double> F, A, Ai;
  CloverIO<PREC_DOUBLE>::load_block(F, a.T64, g.Vh_pad, parity, s, b);
  for (int i = 0; i < 6; i++) A.d[i] = 1.0 + a.csw_eff * F.d[i];
  for (int k = 0; k < 15; k++) A.o[k] = mk(a.csw_eff * F.o[k].re, a.csw_eff * F.o[k].im);
  int st = ldl_invert(A, Ai);
  if (st >= 1 && a.status) atomicAdd(&a.status[0], 1);
  if (st >= 2 && a.status) atomicAdd(&a.status[1], 1);
  if (a.A64) CloverIO<PREC_DOUBLE>::store_block(a.A64, g.Vh_pad, parity, s, b, A, nullptr);
  if (a.Ainv64) CloverIO<PREC_DOUBLE>::store_block(a.Ainv64, g.Vh_pad, parity, s, b, Ai, nullptr);
  if (a.Ainv32) CloverIO<PREC_SINGLE>::store_block(a.Ainv32, g.Vh_pad, parity, s, b, Ai, nullptr);
}

// converts a packed FP64 clover field (both parities) to 16-bit storage
__global__ void clover_to_half_kernel(Geom g, const void* src64, void* dst16) {
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site >= 2 * g.Vh) return;
  const int parity = site >= g.Vh ? 1 : 0;
  const int s = site - parity * g.Vh;
  HermBlock<double> B[2];
  CloverIO<PREC_DOUBLE>::load_block(B[0], src64, g.Vh_pad, parity, s, 0);
  CloverIO<PREC_DOUBLE>::load_block(B[1], src64, g.Vh_pad, parity, s, 1);
  CloverIO<PREC_HALF>::store_site(dst16, g.Vh_pad, parity, s, B);
}

cudaError_t launch_clover_build(const Geom& g, const void* gauge64, double csw_eff, void* A64, void* Ainv64,
                                void* Ainv32, void* Ainv16, int* status, cudaStream_t stream, void* F64, bool F_ready) {
  CloverBuildArgs a;
  a.g = g;
  a.gauge = gauge64;
  a.T64 = F64;
  a.csw_eff = csw_eff;
  a.A64 = A64;
  a.Ainv64 = Ainv64;
  a.Ainv32 = Ainv32;
  a.Ainv16 = Ainv16;
  a.status = status;
  if ((Ainv16 && !Ainv64) || !F64) return cudaErrorInvalidValue;
  if (!F_ready) {
    clover_field_kernel<<<(2 * g.Vh + 31) / 32, dim3(32, 6), 0, stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  clover_assemble_kernel<<<(4 * g.Vh + 127) / 128, 128, 0, stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (Ainv16) {
    clover_to_half_kernel<<<(2 * g.Vh + 127) / 128, 128, 0, stream>>>(g, Ainv64, Ainv16);
    e = cudaGetLastError();
  }
  return e;
}

// out = C in for one parity (C = A or A^-1, any precision), optional norm
template <int P, bool NORM>
__global__ void __launch_bounds__(256) clover_apply_kernel(Geom g, int parity, int nrhs, CSpinorView in, SpinorView out,
                                                           const void* clov, size_t clov_stride, const int* clov_idx,
                                                           const int* active, ReduceArgs red) {
  typedef typename CompReal<P>::type R;
  const int r = blockIdx.y * blockDim.x + threadIdx.x;
  const int s = blockIdx.x * blockDim.y + threadIdx.y;
  const bool valid = (s < g.Vh) && (r < nrhs) && (active == nullptr || active[r]);
  double nrm = 0.0;
  if (valid) {
    Spinor<R> v;
    SpinorIO<P>::load(v, in, s, r);
    const void* c = clov;
    if (clov_idx) c = clov_idx[r] >= 0 ? static_cast<const char*>(clov) + clov_stride * (size_t)clov_idx[r] : nullptr;
    if (c) clover_apply_site<P>(v, c, g.Vh_pad, parity, s);  // negative slot: A = 1
    if (out.data) SpinorIO<P>::store(out, s, r, v);
    if (NORM)
      for (int k = 0; k < 12; k++) nrm += (double)v.c[k].re * v.c[k].re + (double)v.c[k].im * v.c[k].im;
  }
  if (NORM) {
    double vv[1] = {nrm};
    block_reduce_finish<1, FinNone>(vv, nrhs, red);
  }
}

// |A r|^2 (reduced per RHS) and u = A^-1 r from the FP64 r, one read of r.
// PU = PREC_DOUBLE: u in FP64, one chiral block at a time (six components of
// r, one 6x6 block of A, then of A^-1), so a thread holds one block and half a
// spinor. PU = the sloppy precision: u and r rounded to it (the inputs of the
// sloppy-operator r_ne), with the roundings of a separate conversion.
template <int PU, class Fin>
__global__ void __launch_bounds__(256, 2) clover_res_kernel(Geom g, int parity, int nrhs, CSpinorView rin, SpinorView u,
                                                            SpinorView rs, const void* A, const void* Ainv,
                                                            size_t clov_stride, const int* clov_idx, const int* active,
                                                            ReduceArgs red) {
  const int r = blockIdx.y * blockDim.x + threadIdx.x;
  const int s = blockIdx.x * blockDim.y + threadIdx.y;
  const bool valid = (s < g.Vh) && (r < nrhs) && (active == nullptr || active[r]);
  double nrm = 0.0;
  if (valid) {
    const double2* rp = static_cast<const double2*>(rin.data);
    double2* up = static_cast<double2*>(u.data);
    const int ci = clov_idx ? clov_idx[r] : 0;  // negative slot: A = 1
    const char* a = ci >= 0 ? static_cast<const char*>(A) + clov_stride * (size_t)ci : nullptr;
    const char* ai = ci >= 0 ? static_cast<const char*>(Ainv) + clov_stride * (size_t)ci : nullptr;
    typedef typename CompReal<PU>::type RU;
    Spinor<RU> us, rr;  // sloppy outputs (unused for PU = PREC_DOUBLE)
    auto block = [&](const int b) {
      Cplx<double> v[6], w[6];
#pragma unroll
      for (int i = 0; i < 6; i++) {
        const double2 x = rp[chunk_index(6 * b + i, s, r, 12, rin.nrhs)];
        v[i] = w[i] = mk(x.x, x.y);
      }
      if (a) {
        HermBlock<double> B;
        CloverIO<PREC_DOUBLE>::load_block(B, a, g.Vh_pad, parity, s, b);
        herm_apply(B, v);
        CloverIO<PREC_DOUBLE>::load_block(B, ai, g.Vh_pad, parity, s, b);
        herm_apply(B, w);
      }
#pragma unroll
      for (int i = 0; i < 6; i++) {
        nrm = fma(v[i].re, v[i].re, nrm);
        nrm = fma(v[i].im, v[i].im, nrm);
        if constexpr (PU == PREC_DOUBLE) {
          up[chunk_index(6 * b + i, s, r, 12, u.nrhs)] = make_double2(w[i].re, w[i].im);
        } else {
          const double2 x = rp[chunk_index(6 * b + i, s, r, 12, rin.nrhs)];
          us.c[6 * b + i] = mk((RU)w[i].re, (RU)w[i].im);
          rr.c[6 * b + i] = mk((RU)x.x, (RU)x.y);
        }
      }
    };
    if constexpr (PU == PREC_DOUBLE) {
#pragma unroll 1
      for (int b = 0; b < 2; b++) block(b);
    } else {  // unrolled, so that the sloppy spinors stay in registers
      block(0);
      block(1);
    }
    if constexpr (PU != PREC_DOUBLE) {
      SpinorIO<PU>::store(u, s, r, us);
      SpinorIO<PU>::store(rs, s, r, rr);
    }
  }
  double vv[1] = {nrm};
  block_reduce_finish<1, Fin>(vv, nrhs, red);
}

cudaError_t launch_clover_res(int pu, const Geom& g, int parity, int nrhs, CSpinorView r, SpinorView u, SpinorView rs,
                              const void* A, const void* Ainv, size_t clov_stride, const int* clov_idx,
                              const int* active, const ReduceArgs& red, LaunchShape sh, cudaStream_t stream,
                              int fin) {
  dim3 block(sh.Rb, sh.Sb);
  dim3 grid(grid_x(g.Vh, sh.Sb), (nrhs + sh.Rb - 1) / sh.Rb);
  if (fin != FIN_NONE && (fin != FIN_REL_CONT || !red.state)) return cudaErrorInvalidValue;
#define QCU_CR(P)                                                                                                   \
  if (fin == FIN_REL_CONT)                                                                                          \
    clover_res_kernel<P, FinRelCont><<<grid, block, 0, stream>>>(g, parity, nrhs, r, u, rs, A, Ainv, clov_stride,   \
                                                                 clov_idx, active, red);                            \
  else                                                                                                              \
    clover_res_kernel<P, FinNone><<<grid, block, 0, stream>>>(g, parity, nrhs, r, u, rs, A, Ainv, clov_stride,      \
                                                              clov_idx, active, red)
  switch (pu) {
    case PREC_DOUBLE: QCU_CR(PREC_DOUBLE); break;
    case PREC_SINGLE: QCU_CR(PREC_SINGLE); break;
    case PREC_HALF: QCU_CR(PREC_HALF); break;
    default: return cudaErrorInvalidValue;
  }
#undef QCU_CR
  return cudaGetLastError();
}

cudaError_t launch_clover_apply(int prec, const Geom& g, int parity, int nrhs, CSpinorView in, SpinorView out,
                                const void* clov, size_t clov_stride, const int* clov_idx, const int* active,
                                const ReduceArgs* red, LaunchShape sh, cudaStream_t stream) {
  dim3 block(sh.Rb, sh.Sb);
  dim3 grid(grid_x(g.Vh, sh.Sb), (nrhs + sh.Rb - 1) / sh.Rb);
  ReduceArgs rd = red ? *red : ReduceArgs{nullptr, nullptr, nullptr, nullptr};
#define QCU_CL(P)                                                                                             \
  if (red) clover_apply_kernel<P, true><<<grid, block, 0, stream>>>(g, parity, nrhs, in, out, clov, clov_stride, clov_idx, active, rd); \
  else clover_apply_kernel<P, false><<<grid, block, 0, stream>>>(g, parity, nrhs, in, out, clov, clov_stride, clov_idx, active, rd);
  switch (prec) {
    case PREC_DOUBLE: QCU_CL(PREC_DOUBLE) break;
    case PREC_SINGLE: QCU_CL(PREC_SINGLE) break;
    case PREC_HALF: QCU_CL(PREC_HALF) break;
    default: return cudaErrorInvalidValue;
  }
#undef QCU_CL
  return cudaGetLastError();
}

}  // namespace qcu
