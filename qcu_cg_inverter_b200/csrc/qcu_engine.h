// Batch engine of the mixed-precision CG: a fixed set of RHS columns on one
// context (one lattice, one resident gauge field) that right-hand sides join
// and leave between chunks of iterations.
//
// Every kernel of the solver works on all columns under per-column masks
// (qcu_solver.h), so a column can be admitted (source staged, bhat computed,
// x = 0) or retired (x_o reconstructed, solution copied out) while the other
// columns keep iterating; their arithmetic does not depend on which other
// columns are occupied. A step enqueues, without waiting:
//   admissions -> reliable update of the admitted columns -> K sloppy
//   iterations (CUDA graphs) -> reliable update of every column that paused
//   -> copy of the per-column state to pinned host memory -> event.
// The host looks at the state once per step (observe), retires finished
// requests and sizes the next chunk from each column's measured convergence
// rate. qcuInvert drives one engine to completion; the request server
// (server.cu) drives one engine per resident gauge configuration.
#pragma once
#include <vector>

#include "qcu_solver.h"

namespace qcu {

struct EngineParams {
  int precision = PREC_HALF;  // sloppy spinor precision
  double bc_t = -1.0;
  double tol = 1e-10;
  double delta = 0.0;  // 0 = per-precision default
  int maxiter = 20000;
  bool clover = true;  // clover epilogues compiled into the iteration (per-column A = 1 when the slot is -1)
  bool graphs = true;
  // most sloppy iterations per step; new RHS join and finished ones leave only
  // between steps, so a server keeps steps short
  int max_chunk = 64;
  // reliable-update pause alignment (CgDevState::align; 1 = off). Measured:
  // the 48-RHS 24^3x48 batch 0.495 s off, 0.502 s at 8 (its four kappa groups
  // then update more often); the serving stream 288 -> 300 RHS solves/s and
  // p99 2.30 -> 2.00 s at 8
  double align = 1.0;
};

// One request: n consecutive columns with one kappa and one clover slot.
struct Group {
  long long tag = 0;
  int r0 = -1, n = 0;
  double kappa = 0.0;
  int cidx = -1;  // clover slot (-1: A = 1)
  const void* b = nullptr;  // n full AoS spinors (host or device)
  void* x = nullptr;        // n full AoS spinors (host or device)
  bool b_dev = false, x_dev = false;
  enum { QUEUED = 0, ITERATING = 1, RETIRING = 2 };
  int state = QUEUED;
  cudaEvent_t done_ev = nullptr;  // recorded after the solution reached x
  std::vector<qcu_solve_report> reports;
  int status = QCU_SUCCESS;  // worst status of its columns
  Group() = default;
  Group(const Group&) = delete;
  Group& operator=(const Group&) = delete;
  ~Group();
};

class Engine {
 public:
  qcu_context ctx = nullptr;
  int cap = 0;
  EngineParams P;
  SolverWorkspace w;
  DevBuf stage;  // cap full AoS spinors: source in, solution out (per column)
  std::vector<Group*> owner;  // column -> group (nullptr = free)
  std::vector<Group*> pending, live;
  cudaEvent_t step_ev = nullptr;
  bool in_flight = false;
  long long steps = 0;

  ~Engine();
  // (Re)binds to ctx with cap columns; drops every group. Allocates the
  // workspace, captures nothing yet.
  int configure(qcu_context c, int cap, const EngineParams& p);
  int free_columns() const;
  bool idle() const { return live.empty() && pending.empty() && !in_flight; }
  // Takes n free consecutive columns for g (queued until the next step).
  // Returns QCU_ERR_BUSY when no run of g->n free columns exists.
  int admit(Group* g);
  // Enqueues one step; *launched = false when there was nothing to do.
  int step(bool* launched);
  // Non-blocking: true once the last step's state reached the host.
  bool ready();
  int wait();
  // After ready(): updates rates, enqueues the retirement of every group
  // whose columns are all done and appends it to *retired. The group's
  // done_ev fires when its solution is in place.
  int observe(std::vector<Group*>* retired);
  // Drops every group (after an error); columns and clover pins are released.
  void abort();
  long long device_bytes() const;

 private:
  std::vector<int> fresh_;  // admitted in the current step: no state observed yet
  std::vector<double> rate_, seg_rr_;
  std::vector<int> seg_it_, seg_nupd_;
  double prior_rate_ = 0.0;
  RelParams rp_{};
  OpCtx op() const { return OpCtx{ctx, const_cast<SolverWorkspace*>(&w), P.bc_t, ctx->stream}; }
  int enqueue_admissions();
  int enqueue_retirement(const std::vector<Group*>& gs);
  int chunk_length() const;
  void release(Group* g);
};

double default_delta(int precision);

}  // namespace qcu
