// Request server: continuous batching of solves over resident gauge
// configurations (qcuServer* in qcu_b200.h). The reference has no
// counterpart; its only solve entry, cg_inverter (src/cg_inverter.cu:260-369),
// runs one right-hand side at a time to completion.
//
// Each registered configuration becomes resident on first use: a context
// holding its gauge field, a bank of factored clover fields and a batch engine
// with a fixed number of RHS columns. Residency is admitted against a device
// memory budget (configurations with no work are evicted, least recently used
// first, when a new one needs room). A request (kappa, c_sw, nrhs sources) is
// admitted into its configuration's engine as soon as nrhs consecutive
// columns and, for c_sw != 0, a clover slot are free; Wilson requests run in
// the same batch with the clover term switched off for their columns. Every
// engine runs on its own stream, so the batches of different configurations
// overlap on the GPU. The loop (qcuServerPoll) never waits for the GPU: it
// looks at engines whose last step finished, retires finished requests,
// admits queued ones and launches the next step.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "qcu_engine.h"

// reliable-update pause alignment of the server's engines (EngineParams::align).
// Measured on B200 with chunk gathering and delta 2e-3, serving stream (two
// runs each): 1 -> 327.5, 326.9; 3 -> 327.7, 328.6; 8 -> 329.6, 329.0;
// 24 -> 328.6, 327.1 RHS solves/s
#ifndef QCU_SERVER_ALIGN
#define QCU_SERVER_ALIGN 8.0
#endif

using namespace qcu;

extern "C" void qcu_solver_workspace_free(qcu_context ctx);  // engine.cu

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
  long long ticket = 0;
  int config = 0;
  double kappa = 0.0, csw = 0.0;
  int nrhs = 0;
  double t_arrive = 0.0, t_done = 0.0;
  enum { QUEUED = 0, RUNNING = 1, RETIRING = 2, FINISHED = 3 };
  int state = QUEUED;
  Group group;
};

struct Resident {
  int L[4] = {0, 0, 0, 0};
  unsigned long long seed = 0;
  double eps = 0.0;
  qcu_context ctx = nullptr;
  std::unique_ptr<Engine> eng;
  long long bytes = 0;
  long long last_use = 0;
};

}  // namespace

struct qcu_server_s {
  int device = 0;
  qcu_server_params P{};
  long long budget = 0;
  std::vector<Resident> configs;
  std::deque<Request*> queue;
  std::map<long long, std::unique_ptr<Request>> reqs;
  std::vector<Request*> retiring;
  long long next_ticket = 1;
  long long clock = 0;
};

namespace {

// device bytes of a resident configuration (gauge, clover bank, engine)
long long resident_estimate(const qcu_server_params& P, const int L[4]) {
  const Geom g = make_geom(L);
  const int vp = g.Vh_pad, cap = P.columns;
  long long n = 0;
  for (int f : {(int)PREC_DOUBLE, (int)PREC_SINGLE, (int)PREC_HALF, (int)LINK_SINGLE18}) n += gauge_field_bytes(f, vp);
  const long long c16 = (clover_field_bytes(PREC_HALF, vp) + 255) & ~(size_t)255;
  n += (long long)P.clover_slots *
       (2 * (long long)clover_field_bytes(PREC_DOUBLE, vp) + (long long)clover_field_bytes(PREC_SINGLE, vp) + c16);
  n += (long long)clover_field_bytes(PREC_DOUBLE, vp);  // the kappa-independent field term
  const int ps = P.precision, pa = ps == PREC_DOUBLE ? PREC_DOUBLE : PREC_SINGLE;
  n += 9LL * spinor_field_bytes(PREC_DOUBLE, vp, cap);  // b (2 parities), bhat, x, x_o, 4 FP64 temporaries
  n += 2LL * spinor_field_bytes(pa, vp, cap);
  n += 5LL * (spinor_field_bytes(ps, vp, cap) + spinor_norm_bytes(ps, vp, cap));
  n += (long long)cap * 2 * g.Vh * 12 * 16;  // staging of sources and solutions
  n += ((long long)vp * 2 + 1) * cap * 2 * 8 + (64LL << 20);  // reduction scratch, small buffers
  return n;
}

long long resident_bytes(const qcu_server_s* s) {
  long long n = 0;
  for (const Resident& R : s->configs) n += R.ctx ? R.bytes : 0;
  return n;
}

// frees a context without touching the error channel (qcuContextDestroy
// clears it, which would lose the cause of a failed setup)
void destroy_context(qcu_context ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  qcu_solver_workspace_free(ctx);
  delete ctx;
}

void evict(Resident& R) {
  R.eng.reset();
  destroy_context(R.ctx);
  R.ctx = nullptr;
  R.bytes = 0;
}

bool busy(const Resident& R) { return R.eng && !R.eng->idle(); }

long long volume(const int L[4]) { return (long long)L[0] * L[1] * L[2] * L[3]; }

// rank of this lattice among the distinct registered volumes (smallest =
// greatest priority), clamped to the device's priority range
int priority_for(const qcu_server_s* s, const Resident& R) {
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  std::vector<long long> vols;
  for (const Resident& C : s->configs)
    if (std::find(vols.begin(), vols.end(), volume(C.L)) == vols.end()) vols.push_back(volume(C.L));
  std::sort(vols.begin(), vols.end());
  const int rank = (int)(std::find(vols.begin(), vols.end(), volume(R.L)) - vols.begin());
  const int p = greatest + rank;  // greatest is the numerically smallest
  return p > least ? least : p;
}

int make_resident(qcu_server_s* s, int id) {
  Resident& R = s->configs[id];
  if (R.ctx) return QCU_SUCCESS;
  const long long need = resident_estimate(s->P, R.L);
  while (resident_bytes(s) + need > s->budget) {
    int victim = -1;
    for (int k = 0; k < (int)s->configs.size(); k++) {
      const Resident& C = s->configs[k];
      if (C.ctx && !busy(C) && (victim < 0 || C.last_use < s->configs[victim].last_use)) victim = k;
    }
    if (victim < 0) return QCU_ERR_BUSY;  // everything resident is working: wait
    evict(s->configs[victim]);
  }
  qcu_context ctx = nullptr;
  QCU_CHECK(qcuContextCreate(&ctx, R.L, s->device));
  // smaller lattices get higher stream priority: their short kernels are
  // scheduled as soon as SMs free up instead of queueing behind the blocks of
  // large-lattice batches
  int st = ctx_set_stream_priority(ctx, priority_for(s, R));
  if (st == QCU_SUCCESS) st = qcuGenerateGauge(ctx, R.seed, R.eps);
  if (st == QCU_SUCCESS) st = ctx_clover_reserve(ctx, s->P.clover_slots);
  if (st == QCU_SUCCESS && s->P.autotune && !ctx_is_tuned(ctx, ctx_op(ctx, s->P.precision, s->P.columns), s->P.columns))
    st = ctx_autotune(ctx, s->P.precision, s->P.columns, nullptr);
  std::unique_ptr<Engine> eng(new Engine());
  if (st == QCU_SUCCESS) {
    EngineParams ep;
    ep.precision = s->P.precision;
    ep.bc_t = s->P.bc_t;
    ep.tol = s->P.tol;
    ep.delta = s->P.delta;
    ep.maxiter = s->P.maxiter;
    ep.clover = true;
    ep.graphs = true;
    ep.max_chunk = s->P.max_chunk > 0 ? s->P.max_chunk : 8;
    ep.align = QCU_SERVER_ALIGN;
    st = eng->configure(ctx, s->P.columns, ep);
  }
  if (st == QCU_SUCCESS) {
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) st = cuda_status(e, "resident setup");
  }
  if (st != QCU_SUCCESS) {
    eng.reset();
    destroy_context(ctx);
    return st;
  }
  R.ctx = ctx;
  R.bytes = qcuContextDeviceBytes(ctx) + eng->device_bytes();  // the engine is not the context's own
  R.eng = std::move(eng);
  R.last_use = ++s->clock;
  return QCU_SUCCESS;
}

// a clover slot for csw_eff can be had without growing the bank
bool clover_available(qcu_context ctx, double csw_eff) {
  const CloverBank& B = ctx->clover;
  for (int k = 0; k < B.capacity; k++)
    if (B.csw[k] == csw_eff || isnan(B.csw[k]) || B.pinned[k] == 0) return true;
  return false;
}

// QCU_SUCCESS: admitted; QCU_ERR_BUSY: not now; other: the request failed
int try_admit(qcu_server_s* s, Request* q) {
  int st = make_resident(s, q->config);
  if (st != QCU_SUCCESS) return st;
  Resident& R = s->configs[q->config];
  Engine& E = *R.eng;
  if (E.in_flight) return QCU_ERR_BUSY;  // admissions join at step boundaries
  const double csw_eff = q->kappa * q->csw;
  q->group.cidx = -1;
  if (q->csw != 0.0) {
    if (!clover_available(R.ctx, csw_eff)) return QCU_ERR_BUSY;
    // checked for a free run of columns first, so that a slot is not built for nothing
    int run = 0, best = 0;
    for (Group* o : E.owner) {
      run = o ? 0 : run + 1;
      best = run > best ? run : best;
    }
    if (best < q->nrhs) return QCU_ERR_BUSY;
    QCU_CHECK(ctx_clover_slot(R.ctx, csw_eff, &q->group.cidx, false));
  }
  st = E.admit(&q->group);
  if (st != QCU_SUCCESS) return st;
  q->state = Request::RUNNING;
  R.last_use = ++s->clock;
  return QCU_SUCCESS;
}

void finish(qcu_server_s* s, Request* q, double t, int status) {
  q->state = Request::FINISHED;
  q->t_done = t;
  if (status != QCU_SUCCESS && q->group.status == QCU_SUCCESS) q->group.status = status;
  (void)s;
}

}  // namespace

extern "C" {

void qcuServerParamsDefault(qcu_server_params* p) {
  if (!p) return;
  p->precision = QCU_PREC_HALF;
  p->tol = 1e-10;
  p->maxiter = 20000;
  p->bc_t = -1.0;
  p->delta = 0.0;
  p->columns = 16;
  p->clover_slots = 8;
  p->device_budget = 0;
  p->autotune = 1;
  // measured on the 300-request stream: 8 / 16 / 64 give 256 / 253 / 247
  // RHS solves/s and p99 3.15 / 3.25 / 3.42 s
  p->max_chunk = 8;
}

int qcuServerCreate(qcu_server* out, int device, const qcu_server_params* params) {
  clear_error();
  if (!out) {
    set_error(QCU_ERR_INVALID_ARG, "null server handle");
    return QCU_ERR_INVALID_ARG;
  }
  *out = nullptr;
  qcu_server_params P;
  qcuServerParamsDefault(&P);
  if (params) P = *params;
  if (P.columns < 1 || P.columns > 256 || P.clover_slots < 1 || !(P.tol > 0) || P.maxiter < 1 ||
      P.precision < QCU_PREC_DOUBLE || P.precision > QCU_PREC_HALF) {
    set_error(QCU_ERR_INVALID_ARG, "bad server parameters");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK_CUDA(cudaSetDevice(device));
  size_t free_b = 0, total_b = 0;
  QCU_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
  qcu_server_s* s = new qcu_server_s();
  s->device = device;
  s->P = P;
  s->budget = P.device_budget > 0 ? P.device_budget : (long long)(0.85 * (double)free_b);
  *out = s;
  return QCU_SUCCESS;
}

int qcuServerDestroy(qcu_server s) {
  clear_error();
  if (!s) return QCU_SUCCESS;
  for (Resident& R : s->configs) {
    if (R.ctx) cudaStreamSynchronize(R.ctx->stream);
    evict(R);
  }
  delete s;
  return QCU_SUCCESS;
}

int qcuServerAddConfig(qcu_server s, const int lattice[4], unsigned long long seed, double eps, int* config_id) {
  clear_error();
  if (!s || !lattice || !config_id) {
    set_error(QCU_ERR_INVALID_ARG, "bad arguments");
    return QCU_ERR_INVALID_ARG;
  }
  for (int m = 0; m < 4; m++)
    if (lattice[m] < 2 || (m == 0 && lattice[0] % 2)) {
      set_error(QCU_ERR_INVALID_ARG, "bad lattice");
      return QCU_ERR_INVALID_ARG;
    }
  Resident R;
  memcpy(R.L, lattice, sizeof(R.L));
  R.seed = seed;
  R.eps = eps;
  s->configs.push_back(std::move(R));
  *config_id = (int)s->configs.size() - 1;
  return QCU_SUCCESS;
}

int qcuServerPrepare(qcu_server s, int config_id) {
  clear_error();
  if (!s || config_id < 0 || config_id >= (int)s->configs.size()) {
    set_error(QCU_ERR_INVALID_ARG, "unknown configuration");
    return QCU_ERR_INVALID_ARG;
  }
  int st = make_resident(s, config_id);
  if (st == QCU_ERR_BUSY) set_error(st, "device budget exhausted by working configurations");
  return st;
}

int qcuServerSubmit(qcu_server s, int config_id, double kappa, double csw, int nrhs, const void* b, void* x,
                    long long* ticket) {
  clear_error();
  if (!s || !b || !x || !ticket || config_id < 0 || config_id >= (int)s->configs.size() || nrhs < 1 ||
      nrhs > s->P.columns || !(kappa > 0) || !isfinite(kappa) || !isfinite(csw)) {
    set_error(QCU_ERR_INVALID_ARG, "bad request");
    return QCU_ERR_INVALID_ARG;
  }
  std::unique_ptr<Request> q(new Request());
  q->ticket = s->next_ticket++;
  q->config = config_id;
  q->kappa = kappa;
  q->csw = csw;
  q->nrhs = nrhs;
  q->t_arrive = now_s();
  q->group.tag = q->ticket;
  q->group.n = nrhs;
  q->group.kappa = kappa;
  q->group.b = b;
  q->group.x = x;
  q->group.b_dev = is_device_ptr(b);
  q->group.x_dev = is_device_ptr(x);
  *ticket = q->ticket;
  s->queue.push_back(q.get());
  s->reqs[q->ticket] = std::move(q);
  return QCU_SUCCESS;
}

int qcuServerPoll(qcu_server s, int* finished) {
  NvtxRange nv("qcuServerPoll");
  clear_error();
  if (!s) {
    set_error(QCU_ERR_INVALID_ARG, "null server");
    return QCU_ERR_INVALID_ARG;
  }
  int nfin = 0;
  QCU_CHECK_CUDA(cudaSetDevice(s->device));
  // 1. engines whose step finished: observe, retire
  for (Resident& R : s->configs) {
    if (!R.eng || !R.eng->in_flight || !R.eng->ready()) continue;
    std::vector<Group*> ret;
    QCU_CHECK(R.eng->observe(&ret));
    for (Group* g : ret) {
      Request* q = s->reqs[g->tag].get();
      q->state = Request::RETIRING;
      s->retiring.push_back(q);
    }
  }
  // 2. solutions that reached their buffers
  for (size_t i = 0; i < s->retiring.size();) {
    Request* q = s->retiring[i];
    cudaError_t e = cudaEventQuery(q->group.done_ev);
    if (e == cudaErrorNotReady) {
      i++;
      continue;
    }
    if (e != cudaSuccess) return cuda_status(e, "request completion");
    finish(s, q, now_s(), QCU_SUCCESS);
    nfin++;
    s->retiring.erase(s->retiring.begin() + i);
  }
  // 3. admissions, in arrival order; a request that cannot join its batch yet
  //    holds back later requests for the same configuration
  std::vector<char> blocked(s->configs.size(), 0);
  for (size_t i = 0; i < s->queue.size();) {
    Request* q = s->queue[i];
    if (blocked[q->config]) {
      i++;
      continue;
    }
    int st = try_admit(s, q);
    if (st == QCU_SUCCESS) {
      s->queue.erase(s->queue.begin() + i);
    } else if (st == QCU_ERR_BUSY) {
      blocked[q->config] = 1;
      i++;
    } else {  // the request itself cannot run (e.g. singular clover)
      finish(s, q, now_s(), st);
      nfin++;
      s->queue.erase(s->queue.begin() + i);
    }
  }
  // 4. next step of every engine that has work and is not running
  for (Resident& R : s->configs) {
    if (!R.eng || R.eng->in_flight) continue;
    bool launched = false;
    QCU_CHECK(R.eng->step(&launched));
  }
  if (finished) *finished = nfin;
  return QCU_SUCCESS;
}

int qcuServerQuery(qcu_server s, long long ticket, int* finished, double* latency_s, qcu_solve_report* reports) {
  clear_error();
  if (!s || !s->reqs.count(ticket)) {
    set_error(QCU_ERR_INVALID_ARG, "unknown ticket");
    return QCU_ERR_INVALID_ARG;
  }
  Request* q = s->reqs[ticket].get();
  const bool fin = q->state == Request::FINISHED;
  if (finished) *finished = fin ? 1 : 0;
  if (!fin) return QCU_SUCCESS;
  if (latency_s) *latency_s = q->t_done - q->t_arrive;
  if (reports)
    for (int i = 0; i < q->nrhs && i < (int)q->group.reports.size(); i++) reports[i] = q->group.reports[i];
  return q->group.status;
}

int qcuServerRelease(qcu_server s, long long ticket) {
  clear_error();
  if (!s || !s->reqs.count(ticket) || s->reqs[ticket]->state != Request::FINISHED) {
    set_error(QCU_ERR_INVALID_ARG, "unknown or unfinished ticket");
    return QCU_ERR_INVALID_ARG;
  }
  s->reqs.erase(ticket);
  return QCU_SUCCESS;
}

int qcuServerRunTrace(qcu_server s, int n, const double* arrival_s, const int* config_id, const double* kappa,
                      const double* csw, const int* nrhs, const void* const* b, void* const* x, double* latency_s,
                      qcu_solve_report* reports) {
  clear_error();
  if (!s || n < 0 || (n > 0 && (!arrival_s || !config_id || !kappa || !csw || !nrhs || !b || !x || !latency_s))) {
    set_error(QCU_ERR_INVALID_ARG, "bad trace");
    return QCU_ERR_INVALID_ARG;
  }
  for (int i = 1; i < n; i++)
    if (arrival_s[i] < arrival_s[i - 1]) {
      set_error(QCU_ERR_INVALID_ARG, "arrival times must not decrease");
      return QCU_ERR_INVALID_ARG;
    }
  std::vector<long long> tick(n, 0);
  std::vector<size_t> rep_off(n + 1, 0);
  for (int i = 0; i < n; i++) rep_off[i + 1] = rep_off[i] + (size_t)nrhs[i];
  const double t0 = now_s();
  int next = 0, done = 0, ret = QCU_SUCCESS;
  std::vector<char> seen(n, 0);
  while (done < n) {
    const double t = now_s() - t0;
    while (next < n && arrival_s[next] <= t) {
      QCU_CHECK(qcuServerSubmit(s, config_id[next], kappa[next], csw[next], nrhs[next], b[next], x[next], &tick[next]));
      s->reqs[tick[next]]->t_arrive = t0 + arrival_s[next];  // latency counts from the scheduled arrival
      next++;
    }
    int nf = 0;
    QCU_CHECK(qcuServerPoll(s, &nf));
    if (nf == 0) continue;
    for (int i = 0; i < next; i++) {
      if (seen[i]) continue;
      Request* q = s->reqs[tick[i]].get();
      if (q->state != Request::FINISHED) continue;
      seen[i] = 1;
      done++;
      latency_s[i] = q->t_done - q->t_arrive;
      if (reports)
        for (int k = 0; k < q->nrhs && k < (int)q->group.reports.size(); k++) reports[rep_off[i] + k] = q->group.reports[k];
      if (q->group.status != QCU_SUCCESS && ret == QCU_SUCCESS) ret = q->group.status;
      s->reqs.erase(tick[i]);
    }
  }
  if (ret != QCU_SUCCESS) set_error(ret, "not every request reached the tolerance");
  return ret;
}

long long qcuServerDeviceBytes(qcu_server s) { return s ? resident_bytes(s) : 0; }

int qcuServerPending(qcu_server s) {
  if (!s) return 0;
  int n = 0;
  for (auto& kv : s->reqs) n += kv.second->state != Request::FINISHED;
  return n;
}

void* qcuHostAlloc(long long bytes) {
  void* p = nullptr;
  if (bytes <= 0 || cudaHostAlloc(&p, (size_t)bytes, cudaHostAllocDefault) != cudaSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  return p;
}

void qcuHostFree(void* p) {
  if (p) cudaFreeHost(p);
}

}  // extern "C"
