// Batch engine (qcu_engine.h) and qcuInvert on top of it.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "qcu_engine.h"

// Chunk sizing knobs, measured on B200 (16^3x32 solves, kernels per solve):
// predicting exactly (1.0) beats running a quarter ahead (16-bit 375 vs 413,
// FP64 336 vs 391-866), and the last measured rate beats a running mean of
// rates (16-bit 375 every solve vs 363-463).
#ifndef QCU_CHUNK_AHEAD
#define QCU_CHUNK_AHEAD 1.0
#endif
// A chunk runs on past the first predicted trigger to every trigger within
// this fraction of it, so that columns due within a few iterations of one
// another share one reliable-update round and one host round trip (the
// earlier ones pause, masked, meanwhile). The environment variable
// QCU_CHUNK_GATHER overrides it. Measured on B200 at 16-bit delta 2e-3: the
// 48-RHS 24^3x48 batch 0.4616 s (0), 0.4443 s (0.25), 0.4445 s (0.5); the
// serving stream 328.3, 328.5, 327.4 RHS solves/s.
#ifndef QCU_CHUNK_GATHER
#define QCU_CHUNK_GATHER 0.25
#endif
static double chunk_gather() {
  static const double g = [] {
    const char* e = getenv("QCU_CHUNK_GATHER");
    return e ? atof(e) : (double)QCU_CHUNK_GATHER;
  }();
  return g;
}
#ifndef QCU_RATE_SMOOTH
#define QCU_RATE_SMOOTH 0
#endif

namespace qcu {

double default_delta(int precision) {
  // 16-bit inner storage: 2e-3, measured on B200 against 1e-2 and 5e-3 (one
  // reliable update fewer per solve at the same iteration counts): the
  // 16^3x32 solve 3.43 -> 3.26 ms, the 32^3x64 one 28.7 -> 27.3 ms, the
  // serving stream 320 -> 328 RHS solves/s, and with the chunk gathering
  // above the 48-RHS 24^3x48 batch 0.446 -> 0.444 s. FP32 inner solves
  // tolerate 1e-3. An FP64 inner solve needs no
  // update before the convergence check (its iterated residual stays within
  // rounding of the true one at the 1e-10 target), so its delta is tiny and
  // only the target trigger fires: the FP64 solve of the 16^3x32 system
  // 6.54 -> 6.06 ms, of the 24^3x48 one 27.5 -> 25.6 ms against delta 1e-3
  return precision == PREC_HALF ? 2e-3 : (precision == PREC_DOUBLE ? 1e-12 : 1e-3);
}

// Resets columns r0 .. r0+n-1: admit = 1 prepares them for a new RHS (the
// select kernel then picks them for their first reliable update, which
// computes r_ne = Mhat^dag bhat and p = r_ne), admit = 0 marks them free.
__global__ void slot_init_kernel(int nrhs, double* dmem, int* imem, int r0, int n, double kappa, int cidx, int admit) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = r0 + i;
  for (int k = 0; k < D_NUM; k++) dmem[(size_t)k * nrhs + r] = 0.0;
  for (int k = 0; k < I_NUM; k++) imem[(size_t)k * nrhs + r] = 0;
  dmem[(size_t)D_RROLD * nrhs + r] = __longlong_as_double(0x7ff0000000000000LL);  // +inf: beta = 0 at the first update
  dmem[(size_t)D_KAPPA * nrhs + r] = kappa;
  dmem[(size_t)D_MK2 * nrhs + r] = -kappa * kappa;
  dmem[(size_t)D_K2 * nrhs + r] = kappa * kappa;
  imem[(size_t)I_CIDX * nrhs + r] = cidx;
  if (admit) {
    imem[(size_t)I_EVENT * nrhs + r] = 1;
    imem[(size_t)I_ADM * nrhs + r] = 1;
  } else {
    imem[(size_t)I_DONE * nrhs + r] = 1;
  }
}

// |b| of the admitted columns from the dot-product result (re<b,b> at
// res[2r]); a source with NaN or Inf ends its column at once.
__global__ void slot_bnorm_kernel(int nrhs, double* dmem, int* imem, const double* res) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs || !imem[(size_t)I_ADM * nrhs + r]) return;
  const double b2 = res[2 * r];
  if (!isfinite(b2)) {
    imem[(size_t)I_STATUS * nrhs + r] = QCU_ERR_INVALID_ARG;
    imem[(size_t)I_DONE * nrhs + r] = 1;
    imem[(size_t)I_EVENT * nrhs + r] = 0;
    dmem[(size_t)D_TRUE * nrhs + r] = b2;
  } else {
    dmem[(size_t)D_BNORM * nrhs + r] = sqrt(b2);
  }
}

// mask[r] = (r0 <= r < r0+n), or-ed into the old mask when keep = 1
__global__ void mask_range_kernel(int* mask, int nrhs, int r0, int n, int keep) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  const int in = (r >= r0 && r < r0 + n) ? 1 : 0;
  mask[r] = keep ? (mask[r] | in) : in;
}

static inline int nb32(int n) { return (n + 31) / 32; }

Engine::~Engine() {
  abort();
  if (step_ev) cudaEventDestroy(step_ev);
}

int Engine::configure(qcu_context c, int cap_, const EngineParams& p) {
  abort();
  ctx = c;
  cap = cap_;
  P = p;
  QCU_CHECK(ws_prepare(ctx, w, cap, P.precision, P.clover, P.align));
  const size_t full_b = (size_t)2 * ctx->g.Vh * 12 * 16;
  QCU_CHECK(stage.ensure(full_b * cap, ctx->stream));
  if (!step_ev) QCU_CHECK_CUDA(cudaEventCreateWithFlags(&step_ev, cudaEventDisableTiming));
  const double delta = (P.delta > 0 && P.delta < 1) ? P.delta : default_delta(P.precision);
  rp_ = RelParams{P.tol, delta * delta, P.maxiter, P.clover ? 1 : 0};
  QCU_CHECK(ws_set_stop(ctx, w, P.tol, P.maxiter));
  const double sig[5] = {P.bc_t, P.tol, delta * delta, (double)P.maxiter, P.clover ? 1.0 : 0.0};
  if (memcmp(sig, w.graph_sig, sizeof(sig)) != 0) {
    w.drop_graphs();
    memcpy(w.graph_sig, sig, sizeof(sig));
  }
  owner.assign(cap, nullptr);
  fresh_.assign(cap, 1);
  rate_.assign(cap, 0.0);
  seg_rr_.assign(cap, 0.0);
  seg_it_.assign(cap, -1);
  seg_nupd_.assign(cap, 0);
  slot_init_kernel<<<nb32(cap), 32, 0, ctx->stream>>>(cap, w.mem.as<double>(), w.di(0), 0, cap, 0.0, -1, 0);
  QCU_CHECK_CUDA(cudaGetLastError());
  ctx->launches++;
  // the host mirror starts as "all columns free" too
  memset(w.hmem.p, 0, w.mem_bytes());
  for (int r = 0; r < cap; r++) w.hi(I_DONE)[r] = 1;
  in_flight = false;
  return QCU_SUCCESS;
}

int Engine::free_columns() const {
  int n = 0;
  for (Group* g : owner) n += g ? 0 : 1;
  return n;
}

int Engine::admit(Group* g) {
  if (!ctx || g->n < 1 || g->n > cap) {
    set_error(QCU_ERR_INVALID_ARG, "request larger than the batch");
    return QCU_ERR_INVALID_ARG;
  }
  int start = -1;
  for (int r = 0, run = 0; r < cap; r++) {
    run = owner[r] ? 0 : run + 1;
    if (run == g->n) {
      start = r - g->n + 1;
      break;
    }
  }
  if (start < 0) return QCU_ERR_BUSY;
  if (!g->done_ev) QCU_CHECK_CUDA(cudaEventCreateWithFlags(&g->done_ev, cudaEventDisableTiming));
  g->r0 = start;
  g->state = Group::QUEUED;
  g->status = QCU_SUCCESS;
  g->reports.assign(g->n, qcu_solve_report{});
  for (int r = start; r < start + g->n; r++) owner[r] = g;
  if (g->cidx >= 0) ctx->clover.pinned[g->cidx] += 1;
  pending.push_back(g);
  return QCU_SUCCESS;
}

void Engine::release(Group* g) {
  for (int r = g->r0; r < g->r0 + g->n && r < cap; r++)
    if (r >= 0 && owner[r] == g) owner[r] = nullptr;
  if (g->cidx >= 0 && g->cidx < (int)ctx->clover.pinned.size() && ctx->clover.pinned[g->cidx] > 0)
    ctx->clover.pinned[g->cidx] -= 1;
}

void Engine::abort() {
  if (!ctx) return;
  for (Group* g : pending) release(g);
  for (Group* g : live) release(g);
  pending.clear();
  live.clear();
  in_flight = false;
}

long long Engine::device_bytes() const {
  long long n = (long long)w.mem.bytes + (long long)stage.bytes;
  for (const Field* f : {&w.b2, &w.bh, &w.xhi, &w.t64, &w.y64, &w.u64, &w.z64, &w.xo, &w.xlo, &w.rlo, &w.p, &w.t,
                         &w.y, &w.u, &w.z})
    n += (long long)f->data.bytes + (long long)f->norm.bytes;
  return n;
}

// Source in, |b|, bhat = A_ee^-1 (b_e + kappa D_eo A_oo^-1 b_o), x = 0 and
// p = 0, for every column admitted since the last step.
int Engine::enqueue_admissions() {
  NvtxRange nv("qcu admissions");
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  const OpCtx o = op();
  const size_t full_c = (size_t)2 * g.Vh * 12;  // complex numbers of one full spinor
  for (Group* q : pending) {
    const void* src = q->b;
    if (!q->b_dev) {
      char* dst = stage.as<char>() + (size_t)q->r0 * full_c * 16;
      QCU_CHECK_CUDA(cudaMemcpyAsync(dst, q->b, (size_t)q->n * full_c * 16, cudaMemcpyHostToDevice, st));
      src = dst;
    }
    for (int p = 0; p < 2; p++)
      QCU_CHECK_CUDA(launch_spinor_in(PREC_DOUBLE, g, q->n, static_cast<const double2*>(src) + p * (full_c / 2),
                                      full_c, w.b2.view(p), st, q->r0));
    slot_init_kernel<<<nb32(q->n), 32, 0, st>>>(cap, w.mem.as<double>(), w.di(0), q->r0, q->n, q->kappa, q->cidx, 1);
    QCU_CHECK_CUDA(cudaGetLastError());
    ctx->launches += 3;
  }
  const int* adm = w.di(I_ADM);
  {
    ReduceArgs ra = red_into(o, ctx->red.result.as<double>(), false);
    if (g.tdd) {  // the sum runs over both parity blocks whole: their ghost slices must hold zeros
      const size_t per = (size_t)12 * 16 * cap;
      for (int p = 0; p < 2; p++)
        QCU_CHECK_CUDA(cudaMemsetAsync(w.b2.data.as<char>() + p * w.b2.parity_bytes() + g.gfwd * per, 0,
                                       (size_t)2 * g.st * per, st));
    }
    QCU_CHECK_CUDA(launch_cdot(PREC_DOUBLE, 2 * g.Vh_pad, cap, w.b2.cview(0), w.b2.cview(0), adm, ra, w.shape, st));
    QCU_CHECK(dd_sum(ctx, ctx->red.result.as<double>(), 2 * cap, st));
    slot_bnorm_kernel<<<nb32(cap), 32, 0, st>>>(cap, w.mem.as<double>(), w.di(0), ctx->red.result.as<double>());
    QCU_CHECK_CUDA(cudaGetLastError());
    ctx->launches += 2;
  }
  {
    DslashArgs a;
    if (P.clover) {
      QCU_CHECK_CUDA(launch_clover_apply(PREC_DOUBLE, g, 1, cap, w.b2.cview(1), w.t64.view(0),
                                         ctx_clover_ptr(ctx, PREC_DOUBLE, true), ctx_clover_stride(ctx, PREC_DOUBLE),
                                         w.di(I_CIDX), adm, nullptr, w.shape, st));
      ctx->launches++;
      a = op_args(o, PREC_DOUBLE, 0, w.t64, w.bh, adm);
    } else {
      a = op_args(o, PREC_DOUBLE, 0, w.b2, w.bh, adm);
      a.in = w.b2.cview(1);
    }
    a.x = w.b2.cview(0);
    a.coef = w.dd(D_KAPPA);
    QCU_CHECK(dsl(o, PREC_DOUBLE, false, P.clover ? (EPI_XPAY | EPI_CPOST) : EPI_XPAY, FIN_NONE, a));
  }
  QCU_CHECK_CUDA(launch_zero(PREC_DOUBLE, g.Vh, cap, w.xhi.view(0), adm, w.shape, st));
  QCU_CHECK_CUDA(launch_zero(w.pa, g.Vh, cap, w.xlo.view(0), adm, w.shape, st));
  QCU_CHECK_CUDA(launch_zero(w.ps, g.Vh, cap, w.p.view(0), adm, w.shape, st));
  ctx->launches += 3;
  for (Group* q : pending) {
    q->state = Group::ITERATING;
    live.push_back(q);
    for (int r = q->r0; r < q->r0 + q->n; r++) fresh_[r] = 1;
  }
  pending.clear();
  return QCU_SUCCESS;
}

// Iterations until the first iterating column is due for its reliable update
// (predicted from its measured rate), capped by the iteration limit.
int Engine::chunk_length() const {
  // chunk length relative to the predicted distance to the first trigger
  // (never past the iteration cap)
  constexpr double kAhead = QCU_CHUNK_AHEAD;
  double need = 1e30;
  bool any = false;
  std::vector<double> dist;
  dist.reserve(cap);
  for (int r = 0; r < cap; r++) {
    const Group* q = owner[r];
    if (!q || q->state != Group::ITERATING) continue;
    double nd;
    const bool restart = fresh_[r] || (w.hi(I_EVENT)[r] && !w.hi(I_DONE)[r]);
    if (restart) {
      // restarts this step: the segment runs from |r_ne|^2 to delta^2 |r_ne|^2
      const double rt = rate_[r] < 0 ? rate_[r] : prior_rate_;
      nd = rt < 0 ? kAhead * log(rp_.delta2) / rt : 4.0;
      nd = std::min(nd, (double)(P.maxiter - (fresh_[r] ? 0 : w.hi(I_ITERS)[r])));
    } else {
      if (w.hi(I_DONE)[r] || !w.hi(I_ACTIVE)[r]) continue;
      const double rr = w.hd(D_RR)[r], tr = w.hd(D_TRIG)[r];
      const double rt = rate_[r] < 0 ? rate_[r] : prior_rate_;
      nd = (rt < 0 && rr > tr && tr > 0) ? kAhead * log(tr / rr) / rt : 4.0;
      nd = std::min(nd, (double)(P.maxiter - w.hi(I_ITERS)[r]));
    }
    need = std::min(need, nd);
    dist.push_back(nd);
    any = true;
  }
  if (!any) return 0;
  const double reach = need * (1.0 + chunk_gather());
  for (double nd : dist)
    if (nd <= reach) need = std::max(need, nd);
  return (int)std::max(1.0, std::min(ceil(need), (double)std::max(1, P.max_chunk)));
}

NvtxRange::NvtxRange(const char* name) { nvtxRangePushA(name); }
NvtxRange::~NvtxRange() { nvtxRangePop(); }

int Engine::step(bool* launched) {
  NvtxRange nv("qcu engine step");
  *launched = false;
  if (pending.empty() && live.empty()) return QCU_SUCCESS;
  if (w.graph_gen != ctx->clover_gen) {  // the clover bank moved
    w.drop_graphs();
    w.graph_gen = ctx->clover_gen;
  }
  const OpCtx o = op();
  const bool admitting = !pending.empty();
  bool others = false;  // iterating columns due for an update
  for (int r = 0; r < cap && !others; r++) {
    const Group* q = owner[r];
    if (q && q->state == Group::ITERATING && !fresh_[r] && !w.hi(I_DONE)[r] &&
        (w.hi(I_EVENT)[r] || w.hi(I_ITERS)[r] >= P.maxiter))
      others = true;
  }
  if (admitting) QCU_CHECK(enqueue_admissions());
  if (admitting && !others) {  // only new columns: their residual is bhat
    QCU_CHECK(replay(o, -2, P.graphs, [&]() -> int { return enqueue_reliable(o, rp_, true, true); }));
  } else if (admitting || others) {
    QCU_CHECK(replay(o, -1, P.graphs, [&]() -> int { return enqueue_reliable(o, rp_, true); }));
  }
  const bool lead = admitting || others;
  const int K = chunk_length();
  static const bool trace = getenv("QCU_TRACE_STEPS") != nullptr;
  if (trace) {
    for (int r = 0; r < cap; r++) {  // the first column of each group
      if (!owner[r] || owner[r]->r0 != r) continue;
      fprintf(stderr, "step %lld K %d lead %d | r %d it %d nupd %d ev %d done %d rr %.3e trig %.3e rate %.4f prior %.4f fresh %d\n",
              (long long)steps, K, (int)lead, r, w.hi(I_ITERS)[r], w.hi(I_NUPD)[r], w.hi(I_EVENT)[r], w.hi(I_DONE)[r],
              w.hd(D_RR)[r], w.hd(D_TRIG)[r], rate_[r], prior_rate_, (int)fresh_[r]);
    }
  }
  if (K > 0) {
    QCU_CHECK(run_chunk(o, K, P.graphs));
    // every column that paused during the chunk gets its update now
    QCU_CHECK(replay(o, -1, P.graphs, [&]() -> int { return enqueue_reliable(o, rp_, true); }));
  }
  QCU_CHECK_CUDA(cudaMemcpyAsync(w.hmem.p, w.mem.p, w.mem_bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  QCU_CHECK_CUDA(cudaEventRecord(step_ev, ctx->stream));
  in_flight = true;
  steps++;
  *launched = true;
  return QCU_SUCCESS;
}

bool Engine::ready() {
  if (!in_flight) return true;
  cudaError_t e = cudaEventQuery(step_ev);
  if (e == cudaErrorNotReady) return false;
  return true;  // errors surface in observe()
}

int Engine::wait() {
  if (!in_flight) return QCU_SUCCESS;
  QCU_CHECK_CUDA(cudaEventSynchronize(step_ev));
  return QCU_SUCCESS;
}

int Engine::observe(std::vector<Group*>* retired) {
  if (in_flight) {
    QCU_CHECK_CUDA(cudaEventQuery(step_ev));
    in_flight = false;
  }
  // convergence rates: log |r|^2 per iteration, measured over at least
  // kMinSpan iterations (single CG iterations fluctuate too much to predict
  // from: FP64 solves fell into one-iteration steps, 816 kernels instead of
  // 336) and clamped to a plausible range
  constexpr int kMinSpan = 3;
  auto measured = [&](int r, double from, double to, int span) {
    double v = log(to / from) / span;
    v = std::min(-0.002, std::max(-4.0, v));
    rate_[r] = (QCU_RATE_SMOOTH && rate_[r] < 0) ? 0.5 * (rate_[r] + v) : v;
    prior_rate_ = rate_[r];
  };
  for (int r = 0; r < cap; r++) {
    const Group* q = owner[r];
    if (!q || q->state != Group::ITERATING) continue;
    // a column that finished in this step: its last update stopped without
    // closing the segment (D_RRPRE is stale), and its rate is no longer
    // needed; measuring it anyway had left a no-progress rate as the prior of
    // the next solve's first chunk (a 64-iteration chunk, mostly masked)
    if (w.hi(I_DONE)[r]) {
      fresh_[r] = 0;
      continue;
    }
    const int it = w.hi(I_ITERS)[r], nupd = w.hi(I_NUPD)[r];
    const double rr = w.hd(D_RR)[r];
    if (fresh_[r]) {
      fresh_[r] = 0;
    } else if (nupd != seg_nupd_[r]) {  // an update closed the segment at rrpre; rr restarted
      const double pre = w.hd(D_RRPRE)[r];
      if (it - seg_it_[r] >= 2 && pre > 0 && seg_rr_[r] > 0 && pre < seg_rr_[r])
        measured(r, seg_rr_[r], pre, it - seg_it_[r]);
    } else if (it - seg_it_[r] >= kMinSpan && rr > 0 && seg_rr_[r] > 0 && rr < seg_rr_[r]) {
      measured(r, seg_rr_[r], rr, it - seg_it_[r]);
    } else {
      continue;  // too little progress to measure: keep the segment's start point
    }
    seg_it_[r] = it;
    seg_rr_[r] = rr;
    seg_nupd_[r] = nupd;
  }
  std::vector<Group*> done;
  for (Group* q : live) {
    if (q->state != Group::ITERATING) continue;
    bool all = true;
    for (int r = q->r0; r < q->r0 + q->n; r++) all &= w.hi(I_DONE)[r] != 0;
    if (!all) continue;
    int worst = QCU_SUCCESS;
    for (int i = 0; i < q->n; i++) {
      const int r = q->r0 + i;
      const int conv = w.hi(I_CONV)[r], stat = w.hi(I_STATUS)[r];
      qcu_solve_report& rep = q->reports[i];
      rep.iterations = w.hi(I_ITERS)[r];
      rep.reliable_updates = w.hi(I_NUPD)[r];
      rep.converged = conv;
      rep.status = conv ? QCU_SUCCESS : (stat != QCU_SUCCESS ? stat : QCU_ERR_NOT_CONVERGED);
      rep.true_residual = w.hd(D_TRUE)[r];
      rep.kappa = q->kappa;
      {
        const int share = cap > 1 ? w.shape.Rb : 1;  // RHS served by one link / clover load
        // the last reliable update stopped the column: it computed no r_ne
        const double per_site = rep.iterations * iteration_bytes(w.op, P.clover, share) +
                                rep.reliable_updates * reliable_update_bytes(w.op, P.clover, share) -
                                (rep.reliable_updates > 0 ? reliable_update_ne_bytes(w.op, P.clover, share) : 0.0) +
                                admit_retire_bytes(P.clover, share);
        rep.gbytes = per_site * ctx->g.Vh * 1e-9;
        rep.seconds = 0.0;
        rep.gbytes_per_s = 0.0;
      }
      if (rep.status != QCU_SUCCESS && (worst == QCU_SUCCESS || rep.status == QCU_ERR_INVALID_ARG)) worst = rep.status;
    }
    q->status = worst;
    done.push_back(q);
  }
  if (done.empty()) return QCU_SUCCESS;
  QCU_CHECK(enqueue_retirement(done));
  for (Group* q : done) {
    q->state = Group::RETIRING;
    release(q);
    live.erase(std::find(live.begin(), live.end(), q));
    if (retired) retired->push_back(q);
  }
  return QCU_SUCCESS;
}

// x_e += x_lo, x_o = A_oo^-1 (b_o + kappa D_oe x_e), both halves out in the
// AoS layout, and the solution copied to the caller's buffer.
int Engine::enqueue_retirement(const std::vector<Group*>& gs) {
  NvtxRange nv("qcu retirement");
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  const OpCtx o = op();
  int* ret = w.di(I_RET);
  for (size_t i = 0; i < gs.size(); i++) {
    mask_range_kernel<<<nb32(cap), 32, 0, st>>>(ret, cap, gs[i]->r0, gs[i]->n, i ? 1 : 0);
    QCU_CHECK_CUDA(cudaGetLastError());
    ctx->launches++;
  }
  QCU_CHECK_CUDA(launch_accumulate(w.pa, g.Vh, cap, w.xhi.view(0), w.xlo.view(0), ret, w.shape, st));
  ctx->launches++;
  {
    DslashArgs a = op_args(o, PREC_DOUBLE, 1, w.xhi, w.xo, ret);
    a.x = w.b2.cview(1);
    a.coef = w.dd(D_KAPPA);
    QCU_CHECK(dsl(o, PREC_DOUBLE, false, P.clover ? (EPI_XPAY | EPI_CPOST) : EPI_XPAY, FIN_NONE, a));
  }
  const size_t full_c = (size_t)2 * g.Vh * 12;
  for (Group* q : gs) {
    double2* dst = q->x_dev ? static_cast<double2*>(q->x) : stage.as<double2>() + (size_t)q->r0 * full_c;
    QCU_CHECK_CUDA(launch_spinor_out(PREC_DOUBLE, g, q->n, w.xhi.cview(0), dst, full_c, st, q->r0));
    QCU_CHECK_CUDA(launch_spinor_out(PREC_DOUBLE, g, q->n, w.xo.cview(0), dst + full_c / 2, full_c, st, q->r0));
    ctx->launches += 2;
    if (!q->x_dev)
      QCU_CHECK_CUDA(cudaMemcpyAsync(q->x, dst, (size_t)q->n * full_c * 16, cudaMemcpyDeviceToHost, st));
    QCU_CHECK_CUDA(cudaEventRecord(q->done_ev, st));
  }
  return QCU_SUCCESS;
}

Group::~Group() {
  if (done_ev) cudaEventDestroy(done_ev);
}

}  // namespace qcu

using namespace qcu;

extern "C" void qcu_solver_workspace_free(qcu_context ctx) {
  if (ctx) {
    delete ctx->engine;
    ctx->engine = nullptr;
  }
}

extern "C" long long qcu_engine_device_bytes(qcu_context ctx) {
  return (ctx && ctx->engine) ? ctx->engine->device_bytes() : 0;
}

extern "C" int qcuInvert(qcu_context ctx, void* x, const void* b, int nrhs, const double* kappas,
                         const qcu_solve_params* params, qcu_solve_report* reports) {
  NvtxRange nv("qcuInvert");
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
  std::vector<double> kap(nrhs);
  for (int r = 0; r < nrhs; r++) {
    kap[r] = kappas ? kappas[r] : P.kappa;
    if (!(kap[r] > 0.0) || !isfinite(kap[r])) {
      set_error(QCU_ERR_INVALID_ARG, "kappa must be positive");
      return QCU_ERR_INVALID_ARG;
    }
  }
  const bool clover = P.csw != 0.0;
  if (clover) {  // room for one factored clover per distinct kappa*c_sw
    std::vector<double> distinct;
    for (double k : kap)
      if (std::find(distinct.begin(), distinct.end(), k * P.csw) == distinct.end()) distinct.push_back(k * P.csw);
    QCU_CHECK(ctx_clover_reserve(ctx, (int)distinct.size()));
  }
  if (P.autotune && !ctx_is_tuned(ctx, ctx_op(ctx, P.precision, nrhs), nrhs))
    QCU_CHECK(ctx_autotune(ctx, P.precision, nrhs, nullptr));
  if (!ctx->engine) ctx->engine = new Engine();
  Engine& E = *ctx->engine;
  // device time of the call (every admission, step and retirement), for the reports
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess) {
    if (t0) cudaEventDestroy(t0);
    return cuda_status(cudaGetLastError(), "cudaEventCreate");
  }
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } ev_guard{t0, t1};
  QCU_CHECK_CUDA(cudaEventRecord(t0, ctx->stream));
  EngineParams ep;
  ep.precision = P.precision;
  ep.bc_t = P.bc_t;
  ep.tol = P.tol;
  ep.delta = P.delta;
  ep.maxiter = P.maxiter;
  ep.clover = clover;
  ep.graphs = P.use_graphs != 0 && dd_graphs_ok(ctx);
  QCU_CHECK(E.configure(ctx, nrhs, ep));
  // one group per run of equal kappa
  const bool bdev = is_device_ptr(b), xdev = is_device_ptr(x);
  const size_t full_c = (size_t)2 * ctx->g.Vh * 12;
  std::vector<std::unique_ptr<Group>> groups;
  int st = QCU_SUCCESS;
  for (int r = 0; r < nrhs && st == QCU_SUCCESS;) {
    int n = 1;
    while (r + n < nrhs && kap[r + n] == kap[r]) n++;
    groups.emplace_back(new Group());
    Group& q = *groups.back();
    q.tag = r;
    q.n = n;
    q.kappa = kap[r];
    q.b = static_cast<const double2*>(b) + (size_t)r * full_c;
    q.x = static_cast<double2*>(x) + (size_t)r * full_c;
    q.b_dev = bdev;
    q.x_dev = xdev;
    if (clover) st = ctx_clover_slot(ctx, kap[r] * P.csw, &q.cidx);
    if (st == QCU_SUCCESS) st = E.admit(&q);  // pins the slot before the next one is built
    r += n;
  }
  std::vector<Group*> retired;
  for (long long guard = 0; st == QCU_SUCCESS && retired.size() < groups.size(); guard++) {
    bool launched = false;
    st = E.step(&launched);
    if (st != QCU_SUCCESS) break;
    if (!launched || guard > 100000000LL) {
      set_error(QCU_ERR_BREAKDOWN, "solver state stalled");
      st = QCU_ERR_BREAKDOWN;
      break;
    }
    st = E.wait();
    if (st == QCU_SUCCESS) st = E.observe(&retired);
  }
  if (st != QCU_SUCCESS) {
    E.abort();
    return st;
  }
  QCU_CHECK_CUDA(cudaEventRecord(t1, ctx->stream));
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  QCU_CHECK_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  double total_gb = 0.0;
  for (auto& q : groups)
    for (int i = 0; i < q->n; i++) total_gb += q->reports[i].gbytes;
  const double secs = ms * 1e-3;
  int ret = QCU_SUCCESS;
  for (auto& q : groups) {
    for (int i = 0; i < q->n; i++) {
      q->reports[i].seconds = secs;
      q->reports[i].gbytes_per_s = secs > 0 ? total_gb / secs : 0.0;
      if (reports) reports[q->tag + i] = q->reports[i];
    }
    if (q->status == QCU_ERR_INVALID_ARG) ret = QCU_ERR_INVALID_ARG;
    else if (q->status != QCU_SUCCESS && ret == QCU_SUCCESS) ret = q->status;
  }
  if (ret == QCU_ERR_INVALID_ARG) set_error(ret, "source contains NaN or Inf");
  else if (ret != QCU_SUCCESS) set_error(ret, "not every right-hand side reached the tolerance");
  return ret;
}
