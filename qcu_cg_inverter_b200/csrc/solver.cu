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
// FP32 arithmetic; or FP64), six fused kernels per iteration, all scalars
// on the device. Chunks of iterations are replayed as CUDA graphs; the host
// looks at the per-RHS state once per chunk.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "qcu_context.h"

namespace qcu {

enum { D_RR = 0, D_RROLD, D_PAP, D_ALPHA, D_BETA, D_TRIG, D_KAPPA, D_MK2, D_RES_R2, D_RES_AR2, D_RES_NE, D_BNORM,
       D_TRUE, D_NUM };
enum { I_ACTIVE = 0, I_EVENT, I_ITERS, I_BREAK, I_CIDX, I_UPD, I_RST, I_DONE, I_CONV, I_STATUS, I_NUPD, I_NUM };

// Reliable-update control, entirely on the device (one thread per RHS), so an
// update needs no host round trip:
//   select: upd = !done && (paused itself || iteration cap reached)
//   decide: after the FP64 residual kernels, per updated RHS either stop
//           (converged / breakdown / cap) or restart the sloppy residual from
//           r_ne with beta = |r_ne|^2/|r_old|^2 and a new trigger.
struct RelParams {
  double tol, delta2;
  int maxiter;
  int clover;
};

__global__ void rel_select_kernel(int nrhs, int* upd, const int* event, const int* done, const int* iters, int maxiter) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  upd[r] = (!done[r] && (event[r] || iters[r] >= maxiter)) ? 1 : 0;
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
  double ne2 = DV(D_RES_NE);
  double bn = DV(D_BNORM);
  double res = bn > 0 ? sqrt(fmax(ar2, 0.0)) / bn : 0.0;
  DV(D_TRUE) = res;
  int stop = 0;
  if (bn == 0.0 || res < P.tol) {
    IV(I_CONV) = 1;
    stop = 1;
  } else if (!isfinite(res) || IV(I_BREAK)) {
    IV(I_STATUS) = QCU_ERR_BREAKDOWN;
    stop = 1;
  } else if (IV(I_ITERS) >= P.maxiter) {
    IV(I_STATUS) = QCU_ERR_NOT_CONVERGED;
    stop = 1;
  }
  if (stop) {
    IV(I_DONE) = 1;
    IV(I_ACTIVE) = 0;
    IV(I_EVENT) = 0;
    return;
  }
  DV(D_BETA) = ne2 / DV(D_RROLD);  // rr_old = +inf before the first update -> beta = 0
  DV(D_RR) = ne2;
  double q = sqrt(fmax(ar2, 1e-300) / fmax(ne2, 1e-300));
  double target = 0.5 * P.tol * bn / q;
  DV(D_TRIG) = fmax(P.delta2 * ne2, target * target);
  IV(I_ACTIVE) = 1;
  IV(I_EVENT) = 0;
  IV(I_RST) = 1;
#undef DV
#undef IV
}

struct SolverWorkspace {
  int nrhs = 0, ps = -1, pa = -1, op = -1;  // spinor, accumulator precision; sloppy operator variant
  int vh_pad = 0;
  bool clover = false;
  Field b2, bh, xhi, t64, y64, u64, z64, xo;
  Field xlo, rlo, p, t, y, u, z;
  DevBuf mem;       // [D_NUM][nrhs] doubles then [I_NUM][nrhs] ints
  DevBuf dstate;    // CgDevState on the device
  PinnedBuf hmem;   // host mirror of mem
  CgDevState st;
  LaunchShape shape{1, 128};
  std::vector<std::pair<int, cudaGraphExec_t>> graphs;
  long long graph_gen = -1;  // clover bank generation the graphs were captured against
  // kernel arguments and choices baked into the captured graphs
  // (bc_t, tol, delta^2, maxiter, clover on/off)
  double graph_sig[5] = {NAN, NAN, NAN, NAN, NAN};
  ~SolverWorkspace() { drop_graphs(); }
  void drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    graphs.clear();
  }
  double* dd(int k) const { return mem.as<double>() + (size_t)k * nrhs; }
  int* di(int k) const { return reinterpret_cast<int*>(mem.as<double>() + (size_t)D_NUM * nrhs) + (size_t)k * nrhs; }
  double* hd(int k) const { return hmem.as<double>() + (size_t)k * nrhs; }
  int* hi(int k) const { return reinterpret_cast<int*>(hmem.as<double>() + (size_t)D_NUM * nrhs) + (size_t)k * nrhs; }
  size_t mem_bytes() const { return (size_t)D_NUM * nrhs * sizeof(double) + (size_t)I_NUM * nrhs * sizeof(int); }
};

static int ws_prepare(qcu_context ctx, SolverWorkspace& w, int nrhs, int ps, bool clover) {
  cudaStream_t st = ctx->stream;
  const int pa = (ps == PREC_DOUBLE) ? PREC_DOUBLE : PREC_SINGLE;
  const int vp = ctx->g.Vh_pad;
  if (w.nrhs != nrhs || w.ps != ps || w.op != ctx_op(ctx, ps) || w.vh_pad != vp || w.graph_gen != ctx->clover_gen) w.drop_graphs();
  w.graph_gen = ctx->clover_gen;
  w.clover = clover;
  LaunchShape sh = ctx_shape(ctx, ctx_op(ctx, ps), nrhs);
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
  w.op = ctx_op(ctx, ps);
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
  QCU_CHECK_CUDA(cudaMemcpyAsync(w.dstate.p, &w.st, sizeof(CgDevState), cudaMemcpyHostToDevice, st));
  QCU_CHECK(ctx->red.ensure(ctx->g, nrhs, st));
  return QCU_SUCCESS;
}

// ---------------------------------------------------------------------------
// building blocks
// ---------------------------------------------------------------------------
struct OpCtx {
  qcu_context ctx;
  SolverWorkspace* w;
  double bc_t;
  cudaStream_t st;
};

static DslashArgs op_args(const OpCtx& o, int prec, int parity, const Field& in, const Field& out, const int* mask) {
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

static int dsl(const OpCtx& o, int prec, bool dag, int epi, int fin, const DslashArgs& a) {
  QCU_CHECK_CUDA(launch_dslash(prec, dag, epi, fin, a, o.w->shape, o.st));
  o.ctx->launches++;
  return QCU_SUCCESS;
}

static ReduceArgs red_into(const OpCtx& o, double* result, bool with_state) {
  ReduceArgs r = o.ctx->red.args(with_state ? o.w->dstate.p : nullptr);
  r.result = result;
  return r;
}

// One sloppy CG iteration (six launches), masked by the active flags.
static int sloppy_iteration(const OpCtx& o) {
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
  // z = y - k^2 D^dag_eo t
  {
    DslashArgs a = op_args(o, ps, 0, w.t, w.z, act);
    a.x = w.y.cview(0);
    a.coef = w.dd(D_MK2);
    QCU_CHECK(dsl(o, ps, true, EPI_XPAY, FIN_NONE, a));
  }
  // x += alpha p, r -= alpha z, rr -> beta
  QCU_CHECK_CUDA(launch_cg_xr(w.pa, w.ps, o.ctx->g.Vh, w.nrhs, w.xlo.view(0), w.rlo.view(0), w.p.cview(0), w.z.cview(0),
                              w.st.alpha, act, red_into(o, o.ctx->red.result.as<double>(), true), w.shape, o.st));
  // p = r + beta p
  QCU_CHECK_CUDA(launch_cg_p(w.pa, w.ps, o.ctx->g.Vh, w.nrhs, w.p.view(0), w.rlo.cview(0), w.st.beta, act, w.shape, o.st));
  o.ctx->launches += 2;
  return QCU_SUCCESS;
}

// FP64 true residual for the RHS in mask `upd`: x_hi += x_lo, r = bhat - Mhat
// x_hi, |r|^2, |A_ee r|^2 (the full-system residual), r_ne = Mhat^dag r and
// |r_ne|^2 (into D_RES_R2, D_RES_AR2, D_RES_NE).
static int reliable_update(const OpCtx& o) {
  SolverWorkspace& w = *o.w;
  const int* upd = w.di(I_UPD);
  const int Vh = o.ctx->g.Vh;
  QCU_CHECK_CUDA(launch_accumulate(w.pa, Vh, w.nrhs, w.xhi.view(0), w.xlo.view(0), upd, w.shape, o.st));
  o.ctx->launches++;
  {
    DslashArgs a = op_args(o, PREC_DOUBLE, 1, w.xhi, w.t64, upd);
    QCU_CHECK(dsl(o, PREC_DOUBLE, false, w.clover ? EPI_CPRE : 0, FIN_NONE, a));
  }
  {
    DslashArgs a = op_args(o, PREC_DOUBLE, 0, w.t64, w.y64, upd);
    a.x = w.xhi.cview(0);
    a.coef = w.dd(D_MK2);
    QCU_CHECK(dsl(o, PREC_DOUBLE, false, w.clover ? (EPI_CPRE | EPI_XPAY) : EPI_XPAY, FIN_NONE, a));
  }
  // r = bhat - Mhat x (in y64)
  QCU_CHECK_CUDA(launch_residual(Vh, w.nrhs, w.y64.view(0), w.bh.cview(0), w.y64.cview(0), upd,
                                 red_into(o, w.dd(D_RES_R2), false), w.shape, o.st));
  o.ctx->launches++;
  if (w.clover) {
    ReduceArgs ra = red_into(o, w.dd(D_RES_AR2), false);
    SpinorView none{nullptr, nullptr, w.nrhs};
    QCU_CHECK_CUDA(launch_clover_apply(PREC_DOUBLE, o.ctx->g, 0, w.nrhs, w.y64.cview(0), none,
                                       ctx_clover_ptr(o.ctx, PREC_DOUBLE, false), ctx_clover_stride(o.ctx, PREC_DOUBLE),
                                       w.di(I_CIDX), upd, &ra, w.shape, o.st));
    QCU_CHECK_CUDA(launch_clover_apply(PREC_DOUBLE, o.ctx->g, 0, w.nrhs, w.y64.cview(0), w.u64.view(0),
                                       ctx_clover_ptr(o.ctx, PREC_DOUBLE, true), ctx_clover_stride(o.ctx, PREC_DOUBLE),
                                       w.di(I_CIDX), upd, nullptr, w.shape, o.st));
    o.ctx->launches += 2;
  }
  {
    DslashArgs a = op_args(o, PREC_DOUBLE, 1, w.clover ? w.u64 : w.y64, w.t64, upd);
    QCU_CHECK(dsl(o, PREC_DOUBLE, true, w.clover ? EPI_CPRE : 0, FIN_NONE, a));
  }
  {
    DslashArgs a = op_args(o, PREC_DOUBLE, 0, w.t64, w.z64, upd);
    a.x = w.y64.cview(0);
    a.coef = w.dd(D_MK2);
    a.red = red_into(o, w.dd(D_RES_NE), false);
    QCU_CHECK(dsl(o, PREC_DOUBLE, true, EPI_XPAY | EPI_NORM, FIN_NONE, a));
  }
  return QCU_SUCCESS;
}

static int pull_state(const OpCtx& o) {
  SolverWorkspace& w = *o.w;
  QCU_CHECK_CUDA(cudaMemcpyAsync(w.hmem.p, w.mem.p, w.mem_bytes(), cudaMemcpyDeviceToHost, o.st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(o.st));
  return QCU_SUCCESS;
}
// The host mirror is edited right after a push, so the copy must have left
// the pinned buffer before this returns.
static int push_state(const OpCtx& o) {
  SolverWorkspace& w = *o.w;
  QCU_CHECK_CUDA(cudaMemcpyAsync(w.mem.p, w.hmem.p, w.mem_bytes(), cudaMemcpyHostToDevice, o.st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(o.st));
  return QCU_SUCCESS;
}

// Replays (capturing on first use) a CUDA graph of the work `enqueue` puts on
// the stream; `key` identifies the sequence, `nlaunch` counts its kernels.
template <class F>
static int replay(const OpCtx& o, int key, bool graphs, long long nlaunch, F enqueue) {
  SolverWorkspace& w = *o.w;
  if (!graphs) return enqueue();
  cudaGraphExec_t exec = nullptr;
  for (auto& g : w.graphs)
    if (g.first == key) exec = g.second;
  if (!exec) {
    long long before = o.ctx->launches;
    QCU_CHECK_CUDA(cudaStreamBeginCapture(o.st, cudaStreamCaptureModeThreadLocal));
    int s = enqueue();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(o.st, &graph);
    if (s != QCU_SUCCESS) {
      if (graph) cudaGraphDestroy(graph);
      return s;
    }
    QCU_CHECK_CUDA(e);
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    QCU_CHECK_CUDA(e);
    w.graphs.push_back({key, exec});
    o.ctx->launches = before;  // counted when replayed
  }
  QCU_CHECK_CUDA(cudaGraphLaunch(exec, o.st));
  o.ctx->launches += nlaunch;
  return QCU_SUCCESS;
}

// K sloppy iterations as a sum of power-of-two graphs (no overshoot)
static int run_chunk(const OpCtx& o, int K, bool graphs) {
  for (int part = 32; part >= 1; part >>= 1) {
    while (K >= part) {
      QCU_CHECK(replay(o, part, graphs, 6LL * part, [&]() -> int {
        for (int k = 0; k < part; k++) QCU_CHECK(sloppy_iteration(o));
        return QCU_SUCCESS;
      }));
      K -= part;
    }
  }
  return QCU_SUCCESS;
}

// select + FP64 residual + decide + restart, all on the device
static int enqueue_reliable(const OpCtx& o, const RelParams& P, bool select) {
  SolverWorkspace& w = *o.w;
  const int nrhs = w.nrhs;
  const int tb = 32, nb = (nrhs + tb - 1) / tb;
  if (select) {
    rel_select_kernel<<<nb, tb, 0, o.st>>>(nrhs, w.di(I_UPD), w.di(I_EVENT), w.di(I_DONE), w.di(I_ITERS), P.maxiter);
    QCU_CHECK_CUDA(cudaGetLastError());
    o.ctx->launches++;
  }
  QCU_CHECK(reliable_update(o));
  rel_decide_kernel<<<nb, tb, 0, o.st>>>(nrhs, w.mem.as<double>(), w.di(0), P);
  QCU_CHECK_CUDA(cudaGetLastError());
  const int Vh = o.ctx->g.Vh;
  QCU_CHECK_CUDA(launch_convert(w.pa, PREC_DOUBLE, Vh, nrhs, w.rlo.view(0), w.z64.cview(0), w.di(I_RST), nullptr,
                                w.shape, o.st));
  QCU_CHECK_CUDA(launch_cg_p(w.pa, w.ps, Vh, nrhs, w.p.view(0), w.rlo.cview(0), w.dd(D_BETA), w.di(I_RST), w.shape, o.st));
  o.ctx->launches += 3;
  return QCU_SUCCESS;
}

}  // namespace qcu

using namespace qcu;

extern "C" void qcu_solver_workspace_free(qcu_context ctx) {
  if (ctx) {
    delete ctx->solver;
    ctx->solver = nullptr;
  }
}

extern "C" int qcuInvert(qcu_context ctx, void* x, const void* b, int nrhs, const double* kappas,
                         const qcu_solve_params* params, qcu_solve_report* reports) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (!x || !b || nrhs < 1 || !params) {
    set_error(QCU_ERR_INVALID_ARG, "bad solve arguments");
    return QCU_ERR_INVALID_ARG;
  }
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  const qcu_solve_params& P = *params;
  if (P.precision < QCU_PREC_DOUBLE || P.precision > QCU_PREC_HALF || !(P.tol > 0) || P.maxiter < 1) {
    set_error(QCU_ERR_INVALID_ARG, "bad solver parameters");
    return QCU_ERR_INVALID_ARG;
  }
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  std::vector<double> kap(nrhs);
  for (int r = 0; r < nrhs; r++) {
    kap[r] = kappas ? kappas[r] : P.kappa;
    if (!(kap[r] > 0.0) || !isfinite(kap[r])) {
      set_error(QCU_ERR_INVALID_ARG, "kappa must be positive");
      return QCU_ERR_INVALID_ARG;
    }
  }
  const bool clover = P.csw != 0.0;
  // clover slots, one per distinct kappa*c_sw
  std::vector<int> cidx(nrhs, 0);
  if (clover) {
    std::vector<double> distinct;
    for (double k : kap)
      if (std::find(distinct.begin(), distinct.end(), k * P.csw) == distinct.end()) distinct.push_back(k * P.csw);
    QCU_CHECK(ctx_clover_reserve(ctx, (int)distinct.size()));
    for (auto& pin : ctx->clover.pinned) pin = 0;
    for (int r = 0; r < nrhs; r++) {
      int slot;
      QCU_CHECK(ctx_clover_slot(ctx, kap[r] * P.csw, &slot));
      ctx->clover.pinned[slot] = 1;
      cidx[r] = slot;
    }
  }
  if (P.autotune && !ctx_is_tuned(ctx, ctx_op(ctx, P.precision), nrhs))
    QCU_CHECK(ctx_autotune(ctx, P.precision, nrhs, nullptr));
  if (!ctx->solver) ctx->solver = new SolverWorkspace();
  SolverWorkspace& w = *ctx->solver;
  QCU_CHECK(ws_prepare(ctx, w, nrhs, P.precision, clover));
  OpCtx o{ctx, &w, P.bc_t, st};

  // host state
  memset(w.hmem.p, 0, w.mem_bytes());
  for (int r = 0; r < nrhs; r++) {
    w.hd(D_KAPPA)[r] = kap[r];
    w.hd(D_MK2)[r] = -kap[r] * kap[r];
    w.hd(D_RROLD)[r] = INFINITY;
    w.hi(I_CIDX)[r] = cidx[r];
    w.hi(I_UPD)[r] = 1;
  }
  QCU_CHECK(push_state(o));

  // source -> internal, |b|^2
  const size_t full_c = (size_t)2 * g.Vh * 12;  // complex numbers of one full spinor
  const void* bsrc = b;
  if (!is_device_ptr(b)) {
    QCU_CHECK(ctx->stage_in.ensure(full_c * 16 * nrhs, st));
    QCU_CHECK_CUDA(cudaMemcpyAsync(ctx->stage_in.p, b, full_c * 16 * nrhs, cudaMemcpyHostToDevice, st));
    bsrc = ctx->stage_in.p;
  }
  for (int p = 0; p < 2; p++) {
    QCU_CHECK_CUDA(launch_spinor_in(PREC_DOUBLE, g, nrhs, static_cast<const double2*>(bsrc) + p * (full_c / 2), full_c,
                                    w.b2.view(p), st));
    ctx->launches++;
  }
  {
    ReduceArgs ra = red_into(o, ctx->red.result.as<double>(), false);
    QCU_CHECK_CUDA(launch_cdot(PREC_DOUBLE, 2 * g.Vh_pad, nrhs, w.b2.cview(0), w.b2.cview(0), nullptr, ra, w.shape, st));
    ctx->launches++;
    QCU_CHECK_CUDA(cudaMemcpyAsync(ctx->red.host.p, ctx->red.result.p, (size_t)nrhs * 2 * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
    QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  }
  for (int r = 0; r < nrhs; r++) {
    double b2 = ctx->red.host.as<double>()[2 * r];
    if (!isfinite(b2)) {
      set_error(QCU_ERR_INVALID_ARG, "source contains NaN or Inf");
      return QCU_ERR_INVALID_ARG;
    }
    w.hd(D_BNORM)[r] = sqrt(b2);
  }
  QCU_CHECK(push_state(o));
  // bhat = A_ee^-1 (b_e + kappa D_eo A_oo^-1 b_o)
  {
    DslashArgs a;
    if (clover) {
      QCU_CHECK_CUDA(launch_clover_apply(PREC_DOUBLE, g, 1, nrhs, w.b2.cview(1), w.t64.view(0),
                                         ctx_clover_ptr(ctx, PREC_DOUBLE, true), ctx_clover_stride(ctx, PREC_DOUBLE),
                                         w.di(I_CIDX), nullptr, nullptr, w.shape, st));
      ctx->launches++;
      a = op_args(o, PREC_DOUBLE, 0, w.t64, w.bh, nullptr);
    } else {
      a = op_args(o, PREC_DOUBLE, 0, w.b2, w.bh, nullptr);
      a.in = w.b2.cview(1);
    }
    a.x = w.b2.cview(0);
    a.coef = w.dd(D_KAPPA);
    QCU_CHECK(dsl(o, PREC_DOUBLE, false, clover ? (EPI_XPAY | EPI_CPOST) : EPI_XPAY, FIN_NONE, a));
  }
  // x = 0; the first update (all RHS) computes r_ne = Mhat^dag bhat and p = r
  QCU_CHECK_CUDA(cudaMemsetAsync(w.xhi.data.p, 0, w.xhi.data.bytes, st));
  QCU_CHECK_CUDA(cudaMemsetAsync(w.xlo.data.p, 0, w.xlo.data.bytes, st));
  QCU_CHECK_CUDA(cudaMemsetAsync(w.p.data.p, 0, w.p.data.bytes, st));
  if (w.p.norm.p) QCU_CHECK_CUDA(cudaMemsetAsync(w.p.norm.p, 0, w.p.norm.bytes, st));

  // default reliable-update factor per inner precision: measured on the
  // 16^3x32 clover system, 16-bit storage converges in the same iteration
  // count with 1e-2 as with 1e-1 at half the FP64 updates; FP32 and FP64
  // inner solves tolerate 1e-3
  const double delta = P.delta > 0 && P.delta < 1 ? P.delta : (P.precision == QCU_PREC_HALF ? 1e-2 : 1e-3);
  RelParams RP{P.tol, delta * delta, P.maxiter, clover ? 1 : 0};
  const bool graphs = P.use_graphs != 0;
  {
    const double sig[5] = {P.bc_t, P.tol, delta * delta, (double)P.maxiter, clover ? 1.0 : 0.0};
    if (memcmp(sig, w.graph_sig, sizeof(sig)) != 0) {
      w.drop_graphs();
      memcpy(w.graph_sig, sig, sizeof(sig));
    }
  }
  QCU_CHECK(enqueue_reliable(o, RP, false));
  QCU_CHECK(pull_state(o));
  // chunk lengths from each RHS's observed convergence rate
  std::vector<double> rate(nrhs, 0.0), last_rr(nrhs, -1.0);
  std::vector<int> last_it(nrhs, -1);
  for (int loop = 0; loop < 10000000; loop++) {
    int n_left = 0, n_iter = 0;
    for (int r = 0; r < nrhs; r++) {
      if (w.hi(I_DONE)[r]) continue;
      n_left++;
      if (w.hi(I_ACTIVE)[r]) n_iter++;
    }
    if (n_left == 0) break;
    if (n_iter > 0) {
      double need = 1e30;
      bool known = false;
      for (int r = 0; r < nrhs; r++) {
        if (w.hi(I_DONE)[r] || !w.hi(I_ACTIVE)[r]) continue;
        double rr = w.hd(D_RR)[r], tr = w.hd(D_TRIG)[r];
        if (rate[r] < 0 && rr > tr) {
          need = fmin(need, log(tr / rr) / rate[r]);
          known = true;
        }
        need = fmin(need, (double)(P.maxiter - w.hi(I_ITERS)[r]));
      }
      int K = known ? (int)ceil(need) : 4;
      K = std::max(1, std::min(K, 64));
      QCU_CHECK(run_chunk(o, K, graphs));
      QCU_CHECK(pull_state(o));
      for (int r = 0; r < nrhs; r++) {
        int it = w.hi(I_ITERS)[r];
        double rr = w.hd(D_RR)[r];
        if (last_it[r] >= 0 && it > last_it[r] && rr > 0 && last_rr[r] > 0 && rr < last_rr[r])
          rate[r] = log(rr / last_rr[r]) / (it - last_it[r]);
        last_it[r] = it;
        last_rr[r] = rr;
      }
    }
    bool any_upd = false, all_upd = true;
    for (int r = 0; r < nrhs; r++) {
      if (w.hi(I_DONE)[r]) continue;
      bool u = w.hi(I_EVENT)[r] || w.hi(I_ITERS)[r] >= P.maxiter;
      any_upd |= u;
      all_upd &= u;
    }
    if (!any_upd && n_iter == 0) {  // cannot happen: a paused RHS always carries its event
      set_error(QCU_ERR_BREAKDOWN, "solver state stalled");
      return QCU_ERR_BREAKDOWN;
    }
    if (any_upd) {
      QCU_CHECK(replay(o, -1, graphs, 0, [&]() -> int { return enqueue_reliable(o, RP, true); }));
      for (int r = 0; r < nrhs; r++)
        if (!w.hi(I_DONE)[r] && (w.hi(I_EVENT)[r] || w.hi(I_ITERS)[r] >= P.maxiter)) last_it[r] = -1;  // rr restarts
      if (all_upd) QCU_CHECK(pull_state(o));  // nothing iterates until the update is known
    }
  }
  // x_e += x_lo (no-op for checked RHS), x_o = A_oo^-1 (b_o + kappa D_oe x_e)
  for (int r = 0; r < nrhs; r++) w.hi(I_UPD)[r] = 1;
  QCU_CHECK(push_state(o));
  QCU_CHECK_CUDA(launch_accumulate(w.pa, g.Vh, nrhs, w.xhi.view(0), w.xlo.view(0), w.di(I_UPD), w.shape, st));
  {
    DslashArgs a = op_args(o, PREC_DOUBLE, 1, w.xhi, w.xo, nullptr);
    a.x = w.b2.cview(1);
    a.coef = w.dd(D_KAPPA);
    QCU_CHECK(dsl(o, PREC_DOUBLE, false, clover ? (EPI_XPAY | EPI_CPOST) : EPI_XPAY, FIN_NONE, a));
  }
  // solution out
  bool xdev = is_device_ptr(x);
  void* xdst = x;
  if (!xdev) {
    QCU_CHECK(ctx->stage_out.ensure(full_c * 16 * nrhs, st));
    xdst = ctx->stage_out.p;
  }
  QCU_CHECK_CUDA(launch_spinor_out(PREC_DOUBLE, g, nrhs, w.xhi.cview(0), xdst, full_c, st));
  QCU_CHECK_CUDA(launch_spinor_out(PREC_DOUBLE, g, nrhs, w.xo.cview(0), static_cast<double2*>(xdst) + full_c / 2,
                                   full_c, st));
  ctx->launches += 3;
  if (!xdev) QCU_CHECK_CUDA(cudaMemcpyAsync(x, xdst, full_c * 16 * nrhs, cudaMemcpyDeviceToHost, st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  QCU_CHECK(pull_state(o));
  int ret = QCU_SUCCESS;
  for (int r = 0; r < nrhs; r++) {
    int conv = w.hi(I_CONV)[r];
    int stat = w.hi(I_STATUS)[r];
    if (reports) {
      reports[r].iterations = w.hi(I_ITERS)[r];
      reports[r].reliable_updates = w.hi(I_NUPD)[r];
      reports[r].converged = conv;
      reports[r].status = conv ? QCU_SUCCESS : (stat != QCU_SUCCESS ? stat : QCU_ERR_NOT_CONVERGED);
      reports[r].true_residual = w.hd(D_TRUE)[r];
      reports[r].kappa = kap[r];
    }
    if (!conv && ret == QCU_SUCCESS) ret = stat != QCU_SUCCESS ? stat : QCU_ERR_NOT_CONVERGED;
  }
  if (ret != QCU_SUCCESS) set_error(ret, "not every right-hand side reached the tolerance");
  return ret;
}
