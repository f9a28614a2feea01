// Internal interface of the CG solver: device state layout, the workspace of
// one batch of right-hand sides, and the enqueue-only building blocks that
// the batch engine (engine.cu) sequences. solver.cu states the algorithm.
#pragma once
#include <math.h>
#include <string.h>

#include <vector>

#include "qcu_context.h"

namespace qcu {

// Per-RHS device state: D_NUM arrays of doubles then I_NUM arrays of ints,
// each nrhs long (SolverWorkspace::mem); the host mirror has the same layout.
// D_RRPRE: the iterated |r|^2 just before the last reliable update (the end
// point of the convergence segment it closed).
enum { D_RR = 0, D_RROLD, D_PAP, D_ALPHA, D_BETA, D_TRIG, D_KAPPA, D_MK2, D_K2, D_RES_R2, D_RES_AR2, D_RES_NE,
       D_BNORM, D_TRUE, D_RRPRE, D_NUM };  // D_MK2 = -kappa^2, D_K2 = +kappa^2
// I_ADM: RHS being admitted (source staged, bhat and x = 0 to be set up);
// I_RET: RHS being retired (solution reconstructed and copied out).
// I_CONT: RHS of the current reliable update that go on iterating (the others
// stop at it and need no r_ne).
enum { I_ACTIVE = 0, I_EVENT, I_ITERS, I_BREAK, I_CIDX, I_UPD, I_RST, I_DONE, I_CONV, I_STATUS, I_NUPD, I_ADM, I_RET, I_FINAL,
       I_CONT, I_NUM };


struct RelParams {
  double tol, delta2;
  int maxiter;
  int clover;
};


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
  struct Graph {
    int key;
    cudaGraphExec_t exec;
    long long nlaunch;  // kernels in the graph
  };
  std::vector<Graph> graphs;
  long long graph_gen = -1;  // clover bank generation the graphs were captured against
  // kernel arguments and choices baked into the captured graphs
  // (bc_t, tol, delta^2, maxiter, clover on/off)
  double graph_sig[5] = {NAN, NAN, NAN, NAN, NAN};
  ~SolverWorkspace() { drop_graphs(); }
  void drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
  }
  double* dd(int k) const { return mem.as<double>() + (size_t)k * nrhs; }
  int* di(int k) const { return reinterpret_cast<int*>(mem.as<double>() + (size_t)D_NUM * nrhs) + (size_t)k * nrhs; }
  double* hd(int k) const { return hmem.as<double>() + (size_t)k * nrhs; }
  int* hi(int k) const { return reinterpret_cast<int*>(hmem.as<double>() + (size_t)D_NUM * nrhs) + (size_t)k * nrhs; }
  size_t mem_bytes() const { return (size_t)D_NUM * nrhs * sizeof(double) + (size_t)I_NUM * nrhs * sizeof(int); }
};


// Algorithmic bytes per site and RHS of the solver's passes (the counting of
// qcuBenchStencil: every neighbour load, link and clover bytes divided by the
// `share` RHS that one load serves): one sloppy iteration of operator variant
// `op` (the four stencils and p = r + beta p), one reliable update, and the
// admission plus retirement of a column.
double iteration_bytes(int op, bool clover, int share);
double reliable_update_bytes(int op, bool clover, int share);
double reliable_update_ne_bytes(int op, bool clover, int share);  // its r_ne part (not in a stopping update)
double admit_retire_bytes(bool clover, int share);

struct OpCtx {
  qcu_context ctx;
  SolverWorkspace* w;
  double bc_t;
  cudaStream_t st;
};


int ws_prepare(qcu_context ctx, SolverWorkspace& w, int nrhs, int ps, bool clover, double align = 1.0);
// The stopping rule of the reliable updates (tolerance, iteration cap) in the
// device copy of the CG state.
int ws_set_stop(qcu_context ctx, SolverWorkspace& w, double tol, int maxiter);
DslashArgs op_args(const OpCtx& o, int prec, int parity, const Field& in, const Field& out, const int* mask);
int dsl(const OpCtx& o, int prec, bool dag, int epi, int fin, const DslashArgs& a);
ReduceArgs red_into(const OpCtx& o, double* result, bool with_state);
int sloppy_iteration(const OpCtx& o);
// fresh: every selected column was just admitted (x = 0)
int reliable_update(const OpCtx& o, bool fresh = false);
int pull_state(const OpCtx& o);
int push_state(const OpCtx& o);
int run_chunk(const OpCtx& o, int K, bool graphs);
int enqueue_reliable(const OpCtx& o, const RelParams& P, bool select, bool fresh = false);

// Replays (capturing on first use) a CUDA graph of the work `enqueue` puts on
// the stream; `key` identifies the sequence. The kernels `enqueue` counts
// while captured are counted again at every replay.
template <class F>
static int replay(const OpCtx& o, int key, bool graphs, F enqueue) {
  SolverWorkspace& w = *o.w;
  if (!graphs) return enqueue();
  const SolverWorkspace::Graph* hit = nullptr;
  for (auto& g : w.graphs)
    if (g.key == key) hit = &g;
  if (!hit) {
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
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    QCU_CHECK_CUDA(e);
    w.graphs.push_back({key, exec, o.ctx->launches - before});
    o.ctx->launches = before;  // counted when replayed
    hit = &w.graphs.back();
  }
  QCU_CHECK_CUDA(cudaGraphLaunch(hit->exec, o.st));
  o.ctx->launches += hit->nlaunch;
  return QCU_SUCCESS;
}

}  // namespace qcu
