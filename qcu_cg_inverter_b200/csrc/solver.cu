// Even-odd preconditioned CG for M = A - kappa*D with mixed precision and
// reliable updates, batched over right-hand sides (each RHS with its own
// kappa, CG scalars and stopping point).
//
// Schur system on the even sites (the reference solves the full lattice with
// a non-Hermitian pseudo-normal operator, src/cg_inverter.cu:260-369 and
// src/qcu_clover_dslash.cu:1044-1049; this is the mathematically consistent
// replacement, with the true adjoint):
//   Mhat      = 1 - kappa^2 A_ee^-1 D_eo A_oo^-1 D_oe
//   Mhat^dag  = 1 - kappa^2 D^dag_eo A_oo^-1 D^dag_oe A_ee^-1
//   bhat      = A_ee^-1 (b_e + kappa D_eo A_oo^-1 b_o)
//   CG on Mhat^dag Mhat x_e = Mhat^dag bhat, then
//   x_o       = A_oo^-1 (b_o + kappa D_oe x_e).
// The full-system residual of that x is exactly A_ee (bhat - Mhat x_e) on the
// even sites and zero on the odd ones, so every reliable update measures the
// true residual |b - M x| / |b| in FP64 and the solve stops on it.
//
// Inner iterations run in the sloppy precision (16-bit or single storage,
// FP32 arithmetic; or FP64), five fused kernels per iteration (four stencils,
// the last of which also updates x and r, and p = r + beta p), all scalars on
// the device. Chunks of iterations are replayed as CUDA graphs; the host looks
// at the per-RHS state once per chunk.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "qcu_solver.h"

namespace qcu {

// Reliable-update control, entirely on the device (one thread per RHS), so an
// update needs no host round trip:
//   select: upd = !done && (paused itself || iteration cap reached)
//   decide: after the FP64 residual kernels, per updated RHS either stop
//           (converged / breakdown / cap) or restart the sloppy residual from
//           r_ne with beta = |r_ne|^2/|r_old|^2 and a new trigger.
// (select also closes an admission: the admitted RHS carry event = 1)
__global__ void rel_select_kernel(int nrhs, int* upd, const int* event, const int* done, const int* iters, int maxiter,
                                  int* adm) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  upd[r] = (!done[r] && (event[r] || iters[r] >= maxiter)) ? 1 : 0;
  adm[r] = 0;
}

__global__ void rel_decide_kernel(int nrhs, double* dmem, int* imem, RelParams P) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  double* D = dmem;
  int* I = imem;
#define DV(k) D[(size_t)(k) * nrhs + r]
#define IV(k) I[(size_t)(k) * nrhs + r]
  IV(I_RST) = 0;
  if (!IV(I_UPD)) return;
  IV(I_NUPD) += 1;
  double ar2 = P.clover ? DV(D_RES_AR2) : DV(D_RES_R2);
  double ne2 = DV(D_RES_NE);  // computed only for the RHS that go on (I_CONT)
  double bn = DV(D_BNORM);
  double res = 0.0;
  const int why = rel_stop(ar2, bn, IV(I_BREAK), IV(I_ITERS), P.tol, P.maxiter, &res);
  DV(D_TRUE) = res;
  if (why == REL_CONV) IV(I_CONV) = 1;
  else if (why == REL_BREAK) IV(I_STATUS) = QCU_ERR_BREAKDOWN;
  else if (why == REL_CAP) IV(I_STATUS) = QCU_ERR_NOT_CONVERGED;
  if (why != REL_GO) {
    IV(I_DONE) = 1;
    IV(I_ACTIVE) = 0;
    IV(I_EVENT) = 0;
    return;
  }
  DV(D_BETA) = ne2 / DV(D_RROLD);  // rr_old = +inf before the first update -> beta = 0
  DV(D_RRPRE) = DV(D_RR);
  DV(D_RR) = ne2;
  double q = sqrt(fmax(ar2, 1e-300) / fmax(ne2, 1e-300));
  double target = 0.5 * P.tol * bn / q;
  DV(D_TRIG) = fmax(P.delta2 * ne2, target * target);
  IV(I_FINAL) = target * target >= P.delta2 * ne2;  // the next pause is the convergence check
  IV(I_ACTIVE) = 1;
  IV(I_EVENT) = 0;
  IV(I_RST) = 1;
#undef DV
#undef IV
}

static double sb_of(int prec) { return prec == PREC_DOUBLE ? 192.0 : (prec == PREC_SINGLE ? 96.0 : 52.0); }
static double lb_of(int fmt) {
  return fmt == PREC_DOUBLE ? 96.0 : (fmt == PREC_SINGLE ? 48.0 : (fmt == PREC_HALF ? 24.0 : 72.0));
}
static double cb_of(int prec) { return prec == PREC_DOUBLE ? 576.0 : (prec == PREC_SINGLE ? 288.0 : 148.0); }

double iteration_bytes(int op, bool clover, int share) {
  const double sb = sb_of(op_spinor_prec(op)), sa = sb_of(acc_prec(op_spinor_prec(op)));
  const double lb = lb_of(op_link_format(op)), cb = clover ? cb_of(op_clover_prec(op)) : 0.0;
  const double hop = 8.0 * sb + 8.0 * lb / share;
  const double k1 = hop + cb / share + sb;             // t = A^-1 D p
  const double k2 = hop + cb / share + 3.0 * sb;       // y, u from t and p
  const double k3 = k1;                                 // t = A^-1 D^dag u
  const double k4 = hop + 2.0 * sb + 4.0 * sa;          // z = y + c D^dag t, x and r updated
  const double k5 = sa + 2.0 * sb;                      // p = r + beta p
  return k1 + k2 + k3 + k4 + k5;
}

double reliable_update_ne_bytes(int op, bool clover, int share) {
  return iteration_bytes(op, clover, share) * 0.5;  // r_ne = Mhat^dag r, sloppy
}

double reliable_update_bytes(int op, bool clover, int share) {
  const double s64 = 192.0, l64 = 96.0, c64 = clover ? 576.0 : 0.0;
  const double hop64 = 8.0 * s64 + 8.0 * l64 / share;
  const double acc = sb_of(acc_prec(op_spinor_prec(op))) + 4.0 * s64;  // x_hi += x_lo, y = bhat - x_hi
  const double res = 2.0 * hop64 + 2.0 * c64 / share + 3.0 * s64;      // r = bhat - Mhat x_hi
  const double cres = s64 + 2.0 * c64 / share + 2.0 * sb_of(op_spinor_prec(op));
  const double ne = reliable_update_ne_bytes(op, clover, share);
  return acc + res + cres + ne;
}

double admit_retire_bytes(bool clover, int share) {
  const double s64 = 192.0, hop64 = 8.0 * s64 + 8.0 * 96.0 / share, c64 = clover ? 576.0 / share : 0.0;
  // in: AoS -> internal (both parities), |b|^2, bhat; out: x_o, both parities to AoS
  return 4.0 * s64 + 2.0 * s64 + (hop64 + c64 + 2.0 * s64) + s64 + (hop64 + c64 + 2.0 * s64) + 4.0 * s64;
}

int ws_prepare(qcu_context ctx, SolverWorkspace& w, int nrhs, int ps, bool clover, double align) {
  cudaStream_t st = ctx->stream;
  const int pa = acc_prec(ps);
  const int vp = ctx->g.Vh_pad;
  if (w.nrhs != nrhs || w.ps != ps || w.op != ctx_op(ctx, ps, nrhs) || w.vh_pad != vp || w.graph_gen != ctx->clover_gen) w.drop_graphs();
  w.graph_gen = ctx->clover_gen;
  w.clover = clover;
  LaunchShape sh = ctx_shape(ctx, ctx_op(ctx, ps, nrhs), nrhs);
  if (sh.Rb != w.shape.Rb || sh.Sb != w.shape.Sb) w.drop_graphs();
  w.shape = sh;
  QCU_CHECK(w.b2.alloc(PREC_DOUBLE, vp, nrhs, 2, st));
  for (Field* f : {&w.bh, &w.xhi, &w.t64, &w.y64, &w.u64, &w.z64, &w.xo}) QCU_CHECK(f->alloc(PREC_DOUBLE, vp, nrhs, 1, st));
  QCU_CHECK(w.xlo.alloc(pa, vp, nrhs, 1, st));
  QCU_CHECK(w.rlo.alloc(pa, vp, nrhs, 1, st));
  for (Field* f : {&w.p, &w.t, &w.y, &w.u, &w.z}) QCU_CHECK(f->alloc(ps, vp, nrhs, 1, st));
  if (w.nrhs != nrhs || !w.mem.p) {
    w.nrhs = nrhs;
    w.mem.release();
    QCU_CHECK(w.mem.ensure(w.mem_bytes(), st));
    QCU_CHECK(w.hmem.ensure(w.mem_bytes()));
    QCU_CHECK(w.dstate.ensure(sizeof(CgDevState), st));
  }
  w.nrhs = nrhs;
  w.ps = ps;
  w.op = ctx_op(ctx, ps, nrhs);
  w.pa = pa;
  w.vh_pad = vp;
  w.st.rr = w.dd(D_RR);
  w.st.rr_old = w.dd(D_RROLD);
  w.st.pAp = w.dd(D_PAP);
  w.st.alpha = w.dd(D_ALPHA);
  w.st.beta = w.dd(D_BETA);
  w.st.trigger = w.dd(D_TRIG);
  w.st.active = w.di(I_ACTIVE);
  w.st.event = w.di(I_EVENT);
  w.st.iters = w.di(I_ITERS);
  w.st.breakdown = w.di(I_BREAK);
  w.st.final_trig = w.di(I_FINAL);
  w.st.align = align;
  w.st.bnorm = w.dd(D_BNORM);
  w.st.upd = w.di(I_UPD);
  w.st.cont = w.di(I_CONT);
  QCU_CHECK_CUDA(cudaMemcpyAsync(w.dstate.p, &w.st, sizeof(CgDevState), cudaMemcpyHostToDevice, st));
  QCU_CHECK(ctx->red.ensure(ctx->g, nrhs, st, w.shape.Sb));
  return QCU_SUCCESS;
}

int ws_set_stop(qcu_context ctx, SolverWorkspace& w, double tol, int maxiter) {
  w.st.tol = tol;
  w.st.maxiter = maxiter;
  QCU_CHECK_CUDA(cudaMemcpyAsync(w.dstate.p, &w.st, sizeof(CgDevState), cudaMemcpyHostToDevice, ctx->stream));
  return QCU_SUCCESS;
}

// ---------------------------------------------------------------------------
// building blocks
// ---------------------------------------------------------------------------
DslashArgs op_args(const OpCtx& o, int prec, int parity, const Field& in, const Field& out, const int* mask) {
  DslashArgs a;
  memset(&a, 0, sizeof(a));
  a.g = o.ctx->g;
  a.parity = parity;
  a.nrhs = o.w->nrhs;
  a.in = in.cview(0);
  a.out = out.view(0);
  a.gauge = ctx_gauge(o.ctx, prec);
  a.clover = ctx_clover_ptr(o.ctx, prec, true);
  a.clover_stride = ctx_clover_stride(o.ctx, prec);
  a.clover_idx = o.w->di(I_CIDX);
  a.bc_t = o.bc_t;
  a.active = mask;
  return a;
}

int dsl(const OpCtx& o, int prec, bool dag, int epi, int fin, const DslashArgs& a) {
  if (!o.ctx->g.tdd) {
    int n = 0;
    QCU_CHECK_CUDA(launch_dslash(prec, dag, epi, fin, a, o.w->shape, o.st, &n));
    o.ctx->launches += n;
    return QCU_SUCCESS;
  }
  // a t-slab: the input's ghost slices from the neighbouring ranks first; the
  // per-RHS sums of the launch are this slab's part, summed over the ranks
  // before the finishing functor runs
  QCU_CHECK(dd_stencil(o.ctx, a, op_spinor_prec(prec), o.w->shape, o.st, [&](const DslashArgs& piece) {
    int n = 0;
    const cudaError_t e = launch_dslash(prec, dag, epi, FIN_NONE, piece, o.w->shape, o.st, &n);
    o.ctx->launches += n;
    return e;
  }));
  if (epi & (EPI_NORM | EPI_CGXR)) {
    QCU_CHECK(dd_sum(o.ctx, a.red.result, a.nrhs, o.st));
    if (fin != FIN_NONE) {
      QCU_CHECK_CUDA(launch_fin(fin, a.red, a.nrhs, o.st));
      o.ctx->launches++;
    }
  }
  return QCU_SUCCESS;
}

template <class Fin>
__global__ void fin_kernel(const ReduceArgs red, int nrhs) {
  Fin::apply(red.result, nrhs, 1, red.state, (int)threadIdx.x, (int)blockDim.x);
}

cudaError_t launch_fin(int fin, const ReduceArgs& red, int nrhs, cudaStream_t st) {
  if (fin == FIN_CG_ALPHA) fin_kernel<FinCgAlpha><<<1, 64, 0, st>>>(red, nrhs);
  else if (fin == FIN_CG_BETA) fin_kernel<FinCgBeta><<<1, 64, 0, st>>>(red, nrhs);
  else if (fin == FIN_REL_CONT) fin_kernel<FinRelCont><<<1, 64, 0, st>>>(red, nrhs);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

ReduceArgs red_into(const OpCtx& o, double* result, bool with_state) {
  ReduceArgs r = o.ctx->red.args(with_state ? o.w->dstate.p : nullptr);
  r.result = result;
  return r;
}

// One sloppy CG iteration (five launches), masked by the active flags.
int sloppy_iteration(const OpCtx& o) {
  SolverWorkspace& w = *o.w;
  const int ps = w.op;  // operator variant of the sloppy stencils
  const int* act = w.st.active;
  // t = A_oo^-1 D_oe p
  {
    DslashArgs a = op_args(o, ps, 1, w.p, w.t, act);
    QCU_CHECK(dsl(o, ps, false, w.clover ? EPI_CPRE : 0, FIN_NONE, a));
  }
  // y = p - k^2 A_ee^-1 D_eo t, u = A_ee^-1 y, pAp = |y|^2 -> alpha
  {
    DslashArgs a = op_args(o, ps, 0, w.t, w.y, act);
    a.x = w.p.cview(0);
    a.out2 = w.u.view(0);
    a.coef = w.dd(D_MK2);
    a.red = red_into(o, o.ctx->red.result.as<double>(), true);
    int epi = w.clover ? (EPI_CPRE | EPI_XPAY | EPI_OUT2 | EPI_NORM) : (EPI_XPAY | EPI_NORM);
    QCU_CHECK(dsl(o, ps, false, epi, FIN_CG_ALPHA, a));
  }
  // t = A_oo^-1 D^dag_oe u
  {
    DslashArgs a = op_args(o, ps, 1, w.clover ? w.u : w.y, w.t, act);
    QCU_CHECK(dsl(o, ps, true, w.clover ? EPI_CPRE : 0, FIN_NONE, a));
  }
  // z = y - k^2 D^dag_eo t, and in the same kernel x += alpha p, r -= alpha z,
  // rr -> beta (z stays in registers)
  {
    DslashArgs a = op_args(o, ps, 0, w.t, w.z, act);
    a.x = w.y.cview(0);
    a.coef = w.dd(D_MK2);
    a.xacc = w.xlo.view(0);
    a.racc = w.rlo.view(0);
    a.pvec = w.p.cview(0);
    a.alpha = w.st.alpha;
    a.red = red_into(o, o.ctx->red.result.as<double>(), true);
    QCU_CHECK(dsl(o, ps, true, EPI_XPAY | EPI_CGXR, FIN_CG_BETA, a));
  }
  // p = r + beta p
  QCU_CHECK_CUDA(launch_cg_p(w.pa, w.ps, o.ctx->g.Vh, w.nrhs, w.p.view(0), w.rlo.cview(0), w.st.beta, act, w.shape, o.st));
  o.ctx->launches += 1;
  return QCU_SUCCESS;
}

// True residual for the RHS in mask `upd`: x_hi += x_lo, then in FP64
// r = bhat - Mhat x_hi, |r|^2 and |A_ee r|^2 (the full-system residual), and
// r_ne = Mhat^dag r with |r_ne|^2 (into D_RES_R2, D_RES_AR2, D_RES_NE; r_ne
// lands in z, of the sloppy precision, or z64 for FP64 inner solves).
int reliable_update(const OpCtx& o, bool fresh) {
  SolverWorkspace& w = *o.w;
  const int* upd = w.di(I_UPD);
  const int Vh = o.ctx->g.Vh;
  // Only just-admitted columns (x = 0), clover epilogues and a sloppy inner
  // solve: r = bhat exactly, so the FP64 operator passes are skipped and the
  // clover pass reads bhat (the same values as the general path).
  const bool from_b = fresh && w.clover && w.ps != PREC_DOUBLE;
  if (!from_b) {
  // x_hi += x_lo and y64 = bhat - x_hi, then r = y64 + kappa^2 A_ee^-1 D_eo
  // A_oo^-1 D_oe x_hi = bhat - Mhat x_hi in place in y64, with |r|^2
  QCU_CHECK_CUDA(launch_accumulate_res(w.pa, Vh, w.nrhs, w.xhi.view(0), w.xlo.view(0), w.bh.cview(0), w.y64.view(0),
                                       upd, w.shape, o.st));
  o.ctx->launches++;
  {
    DslashArgs a = op_args(o, PREC_DOUBLE, 1, w.xhi, w.t64, upd);
    QCU_CHECK(dsl(o, PREC_DOUBLE, false, w.clover ? EPI_CPRE : 0, FIN_NONE, a));
  }
  {
    DslashArgs a = op_args(o, PREC_DOUBLE, 0, w.t64, w.y64, upd);
    a.x = w.y64.cview(0);  // read and overwritten by the same thread, site by site
    a.coef = w.dd(D_K2);
    a.red = red_into(o, w.dd(D_RES_R2), false);
    QCU_CHECK(dsl(o, PREC_DOUBLE, false, w.clover ? (EPI_CPRE | EPI_XPAY | EPI_NORM) : (EPI_XPAY | EPI_NORM), FIN_NONE,
                  a));
  }
  }
  // r_ne = Mhat^dag r only restarts the sloppy recursion (convergence is
  // decided on the FP64 |A_ee r| below), so with sloppy inner precision it is
  // computed by the sloppy operator from r (and A_ee^-1 r) rounded to the
  // sloppy storage; with FP64 inner precision it stays in FP64
  const bool sloppy_ne = w.ps != PREC_DOUBLE;
  const int pn = sloppy_ne ? w.op : PREC_DOUBLE;
  const Field& rin = sloppy_ne ? w.y : w.y64;
  const Field& uin = sloppy_ne ? w.u : w.u64;
  const Field& tn = sloppy_ne ? w.t : w.t64;
  // r_ne goes straight into the iterated residual when that has its storage
  // (the restart then copies nothing; columns that stop are not read again)
  const bool ne_in_place = (sloppy_ne ? w.ps : PREC_DOUBLE) == w.pa;
  const Field& zn = ne_in_place ? w.rlo : (sloppy_ne ? w.z : w.z64);
  // the RHS that go on after this update (I_CONT, by the decide kernel's
  // stopping rule): only they need r_ne. On one slab with clover the residual
  // reduction's finishing functor marks them; otherwise a one-block launch
  // after the (rank-summed) residual.
  const int* cont = w.di(I_CONT);
  const bool cont_in_res = w.clover && !o.ctx->g.tdd;
  if (w.clover) {  // |A_ee r|^2 and u = A_ee^-1 r in one pass (and r, u rounded to the sloppy storage)
    QCU_CHECK_CUDA(launch_clover_res(sloppy_ne ? w.ps : PREC_DOUBLE, o.ctx->g, 0, w.nrhs,
                                     from_b ? w.bh.cview(0) : w.y64.cview(0),
                                     uin.view(0), w.y.view(0), ctx_clover_ptr(o.ctx, PREC_DOUBLE, false),
                                     ctx_clover_ptr(o.ctx, PREC_DOUBLE, true), ctx_clover_stride(o.ctx, PREC_DOUBLE),
                                     w.di(I_CIDX), upd, red_into(o, w.dd(D_RES_AR2), cont_in_res), w.shape, o.st,
                                     cont_in_res ? FIN_REL_CONT : FIN_NONE));
    o.ctx->launches++;
    QCU_CHECK(dd_sum(o.ctx, w.dd(D_RES_AR2), w.nrhs, o.st));
  } else if (sloppy_ne) {
    QCU_CHECK_CUDA(launch_convert(w.ps, PREC_DOUBLE, Vh, w.nrhs, w.y.view(0), w.y64.cview(0), upd, nullptr, w.shape, o.st));
    o.ctx->launches++;
  }
  if (!cont_in_res) {
    QCU_CHECK_CUDA(launch_fin(FIN_REL_CONT, red_into(o, w.dd(w.clover ? D_RES_AR2 : D_RES_R2), true), w.nrhs, o.st));
    o.ctx->launches++;
  }
  {
    DslashArgs a = op_args(o, pn, 1, w.clover ? uin : rin, tn, cont);
    QCU_CHECK(dsl(o, pn, true, w.clover ? EPI_CPRE : 0, FIN_NONE, a));
  }
  {
    DslashArgs a = op_args(o, pn, 0, tn, zn, cont);
    a.x = rin.cview(0);
    a.coef = w.dd(D_MK2);
    a.red = red_into(o, w.dd(D_RES_NE), false);
    QCU_CHECK(dsl(o, pn, true, EPI_XPAY | EPI_NORM, FIN_NONE, a));
  }
  return QCU_SUCCESS;
}

int pull_state(const OpCtx& o) {
  SolverWorkspace& w = *o.w;
  QCU_CHECK_CUDA(cudaMemcpyAsync(w.hmem.p, w.mem.p, w.mem_bytes(), cudaMemcpyDeviceToHost, o.st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(o.st));
  return QCU_SUCCESS;
}
// The host mirror is edited right after a push, so the copy must have left
// the pinned buffer before this returns.
int push_state(const OpCtx& o) {
  SolverWorkspace& w = *o.w;
  QCU_CHECK_CUDA(cudaMemcpyAsync(w.mem.p, w.hmem.p, w.mem_bytes(), cudaMemcpyHostToDevice, o.st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(o.st));
  return QCU_SUCCESS;
}

// K sloppy iterations as a sum of power-of-two graphs (no overshoot)
int run_chunk(const OpCtx& o, int K, bool graphs) {
  for (int part = 32; part >= 1; part >>= 1) {
    while (K >= part) {
      QCU_CHECK(replay(o, part, graphs, [&]() -> int {
        for (int k = 0; k < part; k++) QCU_CHECK(sloppy_iteration(o));
        return QCU_SUCCESS;
      }));
      K -= part;
    }
  }
  return QCU_SUCCESS;
}

// select + FP64 residual + decide + restart, all on the device
int enqueue_reliable(const OpCtx& o, const RelParams& P, bool select, bool fresh) {
  SolverWorkspace& w = *o.w;
  const int nrhs = w.nrhs;
  const int tb = 32, nb = (nrhs + tb - 1) / tb;
  if (select) {
    rel_select_kernel<<<nb, tb, 0, o.st>>>(nrhs, w.di(I_UPD), w.di(I_EVENT), w.di(I_DONE), w.di(I_ITERS), P.maxiter,
                                           w.di(I_ADM));
    QCU_CHECK_CUDA(cudaGetLastError());
    o.ctx->launches++;
  }
  QCU_CHECK(reliable_update(o, fresh));
  rel_decide_kernel<<<nb, tb, 0, o.st>>>(nrhs, w.mem.as<double>(), w.di(0), P);
  QCU_CHECK_CUDA(cudaGetLastError());
  const int Vh = o.ctx->g.Vh;
  const bool sloppy_ne = w.ps != PREC_DOUBLE;  // where reliable_update left r_ne
  if ((sloppy_ne ? w.ps : PREC_DOUBLE) != w.pa) {  // else it is in rlo already
    QCU_CHECK_CUDA(launch_convert(w.pa, sloppy_ne ? w.ps : PREC_DOUBLE, Vh, nrhs, w.rlo.view(0),
                                  sloppy_ne ? w.z.cview(0) : w.z64.cview(0), w.di(I_RST), nullptr, w.shape, o.st));
    o.ctx->launches++;
  }
  QCU_CHECK_CUDA(launch_cg_p(w.pa, w.ps, Vh, nrhs, w.p.view(0), w.rlo.cview(0), w.dd(D_BETA), w.di(I_RST), w.shape, o.st));
  o.ctx->launches += 2;
  return QCU_SUCCESS;
}

}  // namespace qcu
