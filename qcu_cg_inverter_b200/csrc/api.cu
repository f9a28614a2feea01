// C entry points: the reference-compatible interface (include/qcu.h), the
// reference's operator compositions and the context-based extended API
// (include/qcu_b200.h), minus the solver (solver.cu).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "qcu_context.h"

namespace qcu {

// ---------------------------------------------------------------------------
// errors: per-thread last status, never exit()
// ---------------------------------------------------------------------------
static thread_local int t_err = QCU_SUCCESS;
static thread_local std::string t_msg;

void set_error(int code, const std::string& msg) {
  t_err = code;
  t_msg = msg;
}
void clear_error() {
  t_err = QCU_SUCCESS;
  t_msg.clear();
}
int last_error() { return t_err; }

int cuda_status(cudaError_t e, const char* what) {
  int code = (e == cudaErrorMemoryAllocation) ? QCU_ERR_OUT_OF_MEMORY : QCU_ERR_CUDA;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  set_error(code, m);
  return code;
}

// ---------------------------------------------------------------------------
// device memory
// ---------------------------------------------------------------------------
static std::atomic<long long> g_alloc_fail_after{-1};

void set_alloc_fail_after(long long n) { g_alloc_fail_after.store(n); }

cudaError_t dev_alloc(void** p, size_t bytes) {
  long long n = g_alloc_fail_after.load();
  if (n >= 0) {
    if (n == 0) {
      *p = nullptr;
      return cudaErrorMemoryAllocation;  // injected failure (test hook)
    }
    g_alloc_fail_after.store(n - 1);
  }
  return cudaMalloc(p, bytes);
}

int DevBuf::ensure(size_t n, cudaStream_t st) {
  if (n <= bytes && p) return QCU_SUCCESS;
  release();
  if (n == 0) return QCU_SUCCESS;
  void* q = nullptr;
  cudaError_t e = dev_alloc(&q, n);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return cuda_status(e, "cudaMalloc");
  }
  p = q;
  bytes = n;
  QCU_CHECK_CUDA(cudaMemsetAsync(p, 0, n, st));
  return QCU_SUCCESS;
}
void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

int PinnedBuf::ensure(size_t n) {
  if (n <= bytes && p) return QCU_SUCCESS;
  release();
  void* q = nullptr;
  QCU_CHECK_CUDA(cudaMallocHost(&q, n));
  p = q;
  bytes = n;
  memset(p, 0, n);
  return QCU_SUCCESS;
}
void PinnedBuf::release() {
  if (p) cudaFreeHost(p);
  p = nullptr;
  bytes = 0;
}

int Field::alloc(int prec_, int nsites_, int nrhs_, int nparity_, cudaStream_t st) {
  if (prec == prec_ && nsites == nsites_ && nrhs == nrhs_ && nparity == nparity_ && data.p) return QCU_SUCCESS;
  if (!field_index32_ok(nsites_, nrhs_)) {
    set_error(QCU_ERR_INVALID_ARG, "too many right-hand sides for this lattice (a field must hold < 2^32 chunks)");
    return QCU_ERR_INVALID_ARG;
  }
  prec = prec_;
  nsites = nsites_;
  nrhs = nrhs_;
  nparity = nparity_;
  QCU_CHECK(data.ensure(parity_bytes() * nparity, st));
  if (prec == PREC_HALF) QCU_CHECK(norm.ensure(parity_norm_bytes() * nparity, st));
  return QCU_SUCCESS;
}

SpinorView Field::view(int parity) const {
  SpinorView v;
  v.data = static_cast<char*>(data.p) + parity_bytes() * parity;
  v.norm = prec == PREC_HALF ? reinterpret_cast<float*>(static_cast<char*>(norm.p) + parity_norm_bytes() * parity) : nullptr;
  v.nrhs = nrhs;
  return v;
}

int Scratch::ensure(const Geom& g, int nrhs, cudaStream_t st, int min_sb) {
  // partials: one per (rhs, quantity <= 2, block) for up to 2*Vh_pad sites
  // (full-spinor dot products) in blocks of at least min_sb site lanes
  if (min_sb < 1) min_sb = 1;
  const size_t tiles = (size_t)((g.Vh_pad * 2 + min_sb - 1) / min_sb + 1);
  const size_t groups = (tiles + kReduceGroup - 1) / kReduceGroup + 1;
  size_t need = tiles * (size_t)nrhs * 2;
  if (need > partial_doubles || !partial.p) {
    QCU_CHECK(partial.ensure(need * sizeof(double), st));
    partial_doubles = need;
  }
  // second-level partials and the groups' counters (RHS tiles <= nrhs)
  QCU_CHECK(partial2.ensure(groups * (size_t)nrhs * 2 * sizeof(double), st));
  QCU_CHECK(group_ticket.ensure(groups * (size_t)nrhs * sizeof(unsigned), st));
  QCU_CHECK(ticket.ensure(64, st));
  QCU_CHECK(result.ensure((size_t)nrhs * 2 * sizeof(double) + 64, st));
  QCU_CHECK(host.ensure((size_t)nrhs * 2 * sizeof(double) + 64));
  return QCU_SUCCESS;
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool is_device_ptr_on(const void* p, int device) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == device);
}

// ---------------------------------------------------------------------------
// context helpers
// ---------------------------------------------------------------------------
int ctx_check(qcu_context ctx) {
  if (!ctx) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no context");
    return QCU_ERR_NOT_INITIALIZED;
  }
  QCU_CHECK_CUDA(cudaSetDevice(ctx->device));
  return QCU_SUCCESS;
}

const void* ctx_gauge(qcu_context ctx, int op) {
  switch (op_link_format(op)) {
    case PREC_DOUBLE: return ctx->gauge64.p;
    case PREC_SINGLE: return ctx->gauge32.p;
    case PREC_HALF: return ctx->gauge16.p;
    default: return ctx->gauge18.p;
  }
}

int ingest_gauge(qcu_context ctx, const void* gauge) {
  if (ctx->g.tdd) return dd_ingest_gauge(ctx, gauge);
  const Geom& g = ctx->g;
  QCU_CHECK(ctx->gauge64.ensure(gauge_field_bytes(PREC_DOUBLE, g.Vh_pad), ctx->stream));
  QCU_CHECK(ctx->gauge32.ensure(gauge_field_bytes(PREC_SINGLE, g.Vh_pad), ctx->stream));
  QCU_CHECK(ctx->gauge16.ensure(gauge_field_bytes(PREC_HALF, g.Vh_pad), ctx->stream));
  QCU_CHECK(ctx->gauge18.ensure(gauge_field_bytes(LINK_SINGLE18, g.Vh_pad), ctx->stream));
  const void* src = gauge;
  size_t aos_bytes = (size_t)8 * g.Vh * 9 * 16;
  if (!is_device_ptr(gauge)) {
    QCU_CHECK(ctx->stage_in.ensure(aos_bytes, ctx->stream));
    QCU_CHECK_CUDA(cudaMemcpyAsync(ctx->stage_in.p, gauge, aos_bytes, cudaMemcpyHostToDevice, ctx->stream));
    src = ctx->stage_in.p;
  }
  QCU_CHECK_CUDA(launch_gauge_ingest(g, src, ctx->gauge64.p, ctx->gauge32.p, ctx->gauge16.p, ctx->gauge18.p,
                                     ctx->stream));
  ctx->launches++;
  ctx->gauge_loaded = true;
  ctx->gauge_version++;
  // every factored clover belongs to the previous field
  for (auto& c : ctx->clover.csw) c = NAN;
  return QCU_SUCCESS;
}

int ctx_clover_reserve(qcu_context ctx, int nslots) {
  CloverBank& B = ctx->clover;
  if (nslots <= B.capacity) return QCU_SUCCESS;
  const Geom& g = ctx->g;
  size_t b64 = clover_field_bytes(PREC_DOUBLE, g.Vh_pad);
  size_t b32 = clover_field_bytes(PREC_SINGLE, g.Vh_pad);
  size_t b16 = (clover_field_bytes(PREC_HALF, g.Vh_pad) + 255) & ~(size_t)255;
  DevBuf nA64, nAi64, nAi32, nAi16;
  QCU_CHECK(nA64.ensure(b64 * nslots, ctx->stream));
  QCU_CHECK(nAi64.ensure(b64 * nslots, ctx->stream));
  QCU_CHECK(nAi32.ensure(b32 * nslots, ctx->stream));
  QCU_CHECK(nAi16.ensure(b16 * nslots, ctx->stream));
  if (B.capacity > 0) {
    QCU_CHECK_CUDA(cudaMemcpyAsync(nA64.p, B.A64.p, b64 * B.capacity, cudaMemcpyDeviceToDevice, ctx->stream));
    QCU_CHECK_CUDA(cudaMemcpyAsync(nAi64.p, B.Ainv64.p, b64 * B.capacity, cudaMemcpyDeviceToDevice, ctx->stream));
    QCU_CHECK_CUDA(cudaMemcpyAsync(nAi32.p, B.Ainv32.p, b32 * B.capacity, cudaMemcpyDeviceToDevice, ctx->stream));
    QCU_CHECK_CUDA(cudaMemcpyAsync(nAi16.p, B.Ainv16.p, b16 * B.capacity, cudaMemcpyDeviceToDevice, ctx->stream));
    QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  std::swap(B.A64.p, nA64.p); std::swap(B.A64.bytes, nA64.bytes);
  std::swap(B.Ainv64.p, nAi64.p); std::swap(B.Ainv64.bytes, nAi64.bytes);
  std::swap(B.Ainv32.p, nAi32.p); std::swap(B.Ainv32.bytes, nAi32.bytes);
  std::swap(B.Ainv16.p, nAi16.p); std::swap(B.Ainv16.bytes, nAi16.bytes);
  B.b64 = b64;
  B.b32 = b32;
  B.b16 = b16;
  B.csw.resize(nslots, NAN);
  B.stamp.resize(nslots, 0);
  B.pinned.resize(nslots, 0);
  B.capacity = nslots;
  ctx->clover_gen++;  // device addresses changed: captured graphs are stale
  return QCU_SUCCESS;
}

int ctx_clover_slot(qcu_context ctx, double csw_eff, int* slot, bool wait) {
  CloverBank& B = ctx->clover;
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  for (int k = 0; k < B.capacity; k++)
    if (B.csw[k] == csw_eff) {
      B.stamp[k] = ++ctx->clock;
      *slot = k;
      return QCU_SUCCESS;
    }
  int k = -1;
  for (int i = 0; i < B.capacity; i++)
    if (isnan(B.csw[i])) { k = i; break; }
  if (k < 0) {
    long long best = -1;
    for (int i = 0; i < B.capacity; i++)
      if (!B.pinned[i] && (k < 0 || B.stamp[i] < best)) { k = i; best = B.stamp[i]; }
  }
  if (k < 0) {
    QCU_CHECK(ctx_clover_reserve(ctx, B.capacity + 1));
    k = B.capacity - 1;
  }
  if (ctx->ext) {  // a t-slab: built on the extended slab, its slices copied over
    int es = -1;
    QCU_CHECK(ctx_clover_slot(ctx->ext, csw_eff, &es, true));
    QCU_CHECK(dd_clover_from_ext(ctx, es, k));
    QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    B.csw[k] = csw_eff;
    B.stamp[k] = ++ctx->clock;
    *slot = k;
    return QCU_SUCCESS;
  }
  QCU_CHECK(ctx->status.ensure(64, ctx->stream));
  QCU_CHECK_CUDA(cudaMemsetAsync(ctx->status.p, 0, 64, ctx->stream));
  QCU_CHECK(B.F64.ensure(B.b64, ctx->stream));
  const bool F_ready = B.F_version == ctx->gauge_version;
  QCU_CHECK_CUDA(launch_clover_build(ctx->g, ctx->gauge64.p, csw_eff, static_cast<char*>(B.A64.p) + B.b64 * k,
                                     static_cast<char*>(B.Ainv64.p) + B.b64 * k,
                                     static_cast<char*>(B.Ainv32.p) + B.b32 * k,
                                     static_cast<char*>(B.Ainv16.p) + B.b16 * k, ctx->status.as<int>(), ctx->stream,
                                     B.F64.p, F_ready));
  B.F_version = ctx->gauge_version;
  ctx->launches += F_ready ? 2 : 3;
  if (!wait) {
    B.csw[k] = csw_eff;
    B.stamp[k] = ++ctx->clock;
    *slot = k;
    return QCU_SUCCESS;
  }
  int st[2] = {0, 0};
  QCU_CHECK_CUDA(cudaMemcpyAsync(st, ctx->status.p, sizeof(st), cudaMemcpyDeviceToHost, ctx->stream));
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  if (st[1] > 0) {
    set_error(QCU_ERR_SINGULAR_CLOVER, "clover block with a zero or non-finite pivot");
    return QCU_ERR_SINGULAR_CLOVER;
  }
  B.csw[k] = csw_eff;
  B.stamp[k] = ++ctx->clock;
  *slot = k;
  return QCU_SUCCESS;
}

int ctx_set_stream_priority(qcu_context ctx, int priority) {
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  cudaStream_t s = nullptr;
  QCU_CHECK_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, priority));
  cudaStreamDestroy(ctx->stream);
  ctx->stream = s;
  return QCU_SUCCESS;
}

const void* ctx_clover_ptr(qcu_context ctx, int op, bool inverse) {
  CloverBank& B = ctx->clover;
  if (!inverse) return B.A64.p;
  const int pc = op_clover_prec(op);
  return pc == PREC_DOUBLE ? B.Ainv64.p : (pc == PREC_SINGLE ? B.Ainv32.p : B.Ainv16.p);
}
size_t ctx_clover_stride(qcu_context ctx, int op) {
  CloverBank& B = ctx->clover;
  const int pc = op_clover_prec(op);
  return pc == PREC_DOUBLE ? B.b64 : (pc == PREC_SINGLE ? B.b32 : B.b16);
}

// slot-offset clover pointer
static const void* clover_at(qcu_context ctx, int prec, bool inverse, int slot) {
  return static_cast<const char*>(ctx_clover_ptr(ctx, prec, inverse)) + ctx_clover_stride(ctx, prec) * slot;
}

// ---------------------------------------------------------------------------
// stencil helpers on internal FP64 fields (one RHS)
// ---------------------------------------------------------------------------
static DslashArgs base_args(qcu_context ctx, int prec) {
  DslashArgs a;
  memset(&a, 0, sizeof(a));
  a.g = ctx->g;
  a.nrhs = 1;
  a.gauge = ctx_gauge(ctx, prec);
  a.coef0 = 0.0;
  a.bc_t = 1.0;
  return a;
}

static int run_dslash(qcu_context ctx, int prec, bool dag, int epi, const DslashArgs& a) {
  if (ctx->g.tdd)  // t-slab: the neighbours' faces, beside the interior
    return dd_stencil(ctx, a, op_spinor_prec(prec), ctx->shape1, ctx->stream, [&](const DslashArgs& piece) {
      ctx->launches++;
      return launch_dslash(prec, dag, epi, FIN_NONE, piece, ctx->shape1, ctx->stream);
    });
  QCU_CHECK_CUDA(launch_dslash(prec, dag, epi, FIN_NONE, a, ctx->shape1, ctx->stream));
  ctx->launches++;
  return QCU_SUCCESS;
}

// copies one AoS full/half spinor (device or host) into an internal FP64 field
static int spinor_to_internal(qcu_context ctx, const void* aos, Field& f, int nparity) {
  const Geom& g = ctx->g;
  size_t half_c = (size_t)g.Vh * 12;  // complex numbers per parity
  QCU_CHECK(f.alloc(PREC_DOUBLE, g.Vh_pad, 1, nparity, ctx->stream));
  const void* src = aos;
  if (!is_device_ptr(aos)) {
    QCU_CHECK(ctx->stage_in.ensure(half_c * 16 * nparity, ctx->stream));
    QCU_CHECK_CUDA(cudaMemcpyAsync(ctx->stage_in.p, aos, half_c * 16 * nparity, cudaMemcpyHostToDevice, ctx->stream));
    src = ctx->stage_in.p;
  }
  for (int p = 0; p < nparity; p++) {
    QCU_CHECK_CUDA(launch_spinor_in(PREC_DOUBLE, g, 1, static_cast<const double2*>(src) + p * half_c, 0, f.view(p),
                                    ctx->stream));
    ctx->launches++;
  }
  return QCU_SUCCESS;
}

static int spinor_from_internal(qcu_context ctx, const Field& f, void* aos, int nparity) {
  const Geom& g = ctx->g;
  size_t half_c = (size_t)g.Vh * 12;
  bool dev = is_device_ptr(aos);
  void* dst = aos;
  if (!dev) {
    QCU_CHECK(ctx->stage_out.ensure(half_c * 16 * nparity, ctx->stream));
    dst = ctx->stage_out.p;
  }
  for (int p = 0; p < nparity; p++) {
    QCU_CHECK_CUDA(launch_spinor_out(f.prec, g, 1, f.cview(p), static_cast<double2*>(dst) + p * half_c, 0, ctx->stream));
    ctx->launches++;
  }
  if (!dev)
    QCU_CHECK_CUDA(cudaMemcpyAsync(aos, ctx->stage_out.p, half_c * 16 * nparity, cudaMemcpyDeviceToHost, ctx->stream));
  return QCU_SUCCESS;
}

// out_p = [x_p +] coef [C] D^(dag) in_{1-p} for both parities of full fields
enum RoundKind { ROUND_CLOVER_HOP = 0, ROUND_NEWFULL = 1, ROUND_FULL = 2 };
static int full_round(qcu_context ctx, int kind, const Field& in, Field& out, bool dag, int slot) {
  for (int p = 0; p < 2; p++) {
    DslashArgs a = base_args(ctx, PREC_DOUBLE);
    a.parity = p;
    a.in = in.cview(1 - p);
    a.out = out.view(p);
    a.x = in.cview(p);
    int epi = 0;
    if (kind == ROUND_CLOVER_HOP) {  // A^-1 D
      epi = EPI_CPRE;
      a.clover = clover_at(ctx, PREC_DOUBLE, true, slot);
    } else if (kind == ROUND_NEWFULL) {  // in - A^-1 D in
      epi = EPI_CPRE | EPI_XPAY;
      a.coef0 = -1.0;
      a.clover = clover_at(ctx, PREC_DOUBLE, true, slot);
    } else {  // A in - D in
      epi = EPI_XPAY | EPI_CX;
      a.coef0 = -1.0;
      a.clover = clover_at(ctx, PREC_DOUBLE, false, slot);
    }
    QCU_CHECK(run_dslash(ctx, PREC_DOUBLE, dag, epi, a));
  }
  return QCU_SUCCESS;
}

// in-place clover apply on both parities of a full FP64 field
static int clover_both(qcu_context ctx, const Field& in, Field& out, bool inverse, int slot) {
  for (int p = 0; p < 2; p++) {
    QCU_CHECK_CUDA(launch_clover_apply(PREC_DOUBLE, ctx->g, p, 1, in.cview(p), out.view(p),
                                       clover_at(ctx, PREC_DOUBLE, inverse, slot), 0, nullptr, nullptr, nullptr,
                                       ctx->shape1, ctx->stream));
    ctx->launches++;
  }
  return QCU_SUCCESS;
}

}  // namespace qcu

using namespace qcu;

qcu_context_s::~qcu_context_s() {
  if (stream) cudaStreamDestroy(stream);
}

// ---------------------------------------------------------------------------
// legacy interface (include/qcu.h): one process-wide context, as in the reference
// ---------------------------------------------------------------------------
static std::mutex g_legacy_mu;
static qcu_context g_legacy = nullptr;

static int legacy_begin(QcuParam* param, void* gauge, qcu_context* out) {
  clear_error();
  if (!g_legacy) {
    set_error(QCU_ERR_NOT_INITIALIZED, "initGridSize() must be called first");
    return QCU_ERR_NOT_INITIALIZED;
  }
  if (param) {
    for (int i = 0; i < 4; i++)
      if (param->lattice_size[i] != g_legacy->L[i]) {
        set_error(QCU_ERR_INVALID_ARG, "lattice size differs from initGridSize()");
        return QCU_ERR_INVALID_ARG;
      }
  }
  QCU_CHECK(ctx_check(g_legacy));
  // the reference works on the default stream: the caller's pending work on
  // it (the kernels that produced the arguments) comes first
  QCU_CHECK(qcuContextSetStream(g_legacy, cudaStreamLegacy));
  if (gauge && (!g_legacy->gauge_loaded || g_legacy->legacy_gauge_src != gauge)) {
    QCU_CHECK(ingest_gauge(g_legacy, gauge));
    g_legacy->legacy_gauge_src = gauge;
  }
  *out = g_legacy;
  return QCU_SUCCESS;
}

static int legacy_finish(qcu_context ctx, int st) {
  if (st != QCU_SUCCESS) return st;
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}

static int valid_lattice(const int L[4]) {
  for (int i = 0; i < 4; i++)
    if (L[i] <= 0) return 0;
  if (L[0] % 2) return 0;
  long long V = (long long)L[0] * L[1] * L[2] * L[3];
  if (V / 2 > (1LL << 30) / 12) return 0;
  return 1;
}

extern "C" {

int qcu_last_error(void) { return last_error(); }
const char* qcu_last_error_string(void) { return t_msg.c_str(); }

void qcuSolveParamsDefault(qcu_solve_params* p) {
  if (!p) return;
  p->kappa = 0.12;
  p->csw = 0.0;
  p->bc_t = -1.0;
  p->tol = 1e-10;
  p->maxiter = 20000;
  p->precision = QCU_PREC_HALF;
  p->delta = 0.0;  // per-precision default (default_delta: 2e-3 for 16-bit, 1e-3 single, 1e-12 double)
  p->use_graphs = 1;
  p->autotune = 1;
}

int qcuContextCreate(qcu_context* out, const int lattice[4], int device) {
  clear_error();
  if (!out || !lattice || !valid_lattice(lattice)) {
    set_error(QCU_ERR_INVALID_ARG, "lattice extents must be positive with Lx even");
    return QCU_ERR_INVALID_ARG;
  }
  int ndev = 0;
  QCU_CHECK_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) {
    set_error(QCU_ERR_INVALID_ARG, "no such device");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK_CUDA(cudaSetDevice(device));
  qcu_context ctx = new qcu_context_s();
  ctx->device = device;
  for (int i = 0; i < 4; i++) ctx->L[i] = lattice[i];
  ctx->g = make_geom(lattice);
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ctx;
    return cuda_status(e, "cudaStreamCreate");
  }
  int st = ctx->red.ensure(ctx->g, 1, ctx->stream, ctx->shape1.Sb);
  if (st != QCU_SUCCESS) {
    delete ctx;
    return st;
  }
  e = prepare_staged_kernels();
  if (e != cudaSuccess) {
    qcuContextDestroy(ctx);
    return cuda_status(e, "staged stencil set-up");
  }
  // qcuDslashNoAlloc's device set-up happens here, so that its calls take no
  // device memory; a failure is reported by that entry point, not here
  if (noalloc_prepare(device) != QCU_SUCCESS) clear_error();
  *out = ctx;
  return QCU_SUCCESS;
}

extern "C" void qcu_solver_workspace_free(qcu_context ctx);  // engine.cu
extern "C" long long qcu_engine_device_bytes(qcu_context ctx);

int qcuContextDestroy(qcu_context ctx) {
  clear_error();
  if (!ctx) return QCU_SUCCESS;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  qcu_solver_workspace_free(ctx);
  if (ctx->ext) qcuContextDestroy(ctx->ext);
  if (ctx->dd_stream) {
    cudaStreamSynchronize(ctx->dd_stream);
    cudaStreamDestroy(ctx->dd_stream);
  }
  for (cudaEvent_t e : ctx->dd_ev)
    if (e) cudaEventDestroy(e);
  delete ctx;
  return QCU_SUCCESS;
}

int qcuContextSetStream(qcu_context ctx, void* stream) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  // the context keeps its own stream and orders it after the caller's
  cudaEvent_t ev;
  QCU_CHECK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  QCU_CHECK_CUDA(cudaEventRecord(ev, static_cast<cudaStream_t>(stream)));
  QCU_CHECK_CUDA(cudaStreamWaitEvent(ctx->stream, ev, 0));
  cudaEventDestroy(ev);
  return QCU_SUCCESS;
}

void* qcuContextGetStream(qcu_context ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int qcuContextSetShape(qcu_context ctx, int rhs_lanes, int site_lanes) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  int n = rhs_lanes * site_lanes;
  if (rhs_lanes < 1 || rhs_lanes > 32 || 32 % rhs_lanes || site_lanes < 1 || n % 32 || n > 256) {
    set_error(QCU_ERR_INVALID_ARG, "block shape must have a power-of-two RHS width <= 32 and 32..256 threads");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK(ctx->red.ensure(ctx->g, 1, ctx->stream, site_lanes));
  ctx->shape1 = LaunchShape{rhs_lanes, site_lanes};
  ctx->shape_set = true;
  return QCU_SUCCESS;
}

int qcuContextSetHalfOperator(qcu_context ctx, int fast_links) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  ctx->half_op = fast_links < 0 ? -1 : (fast_links ? OP_HALF_FAST : OP_HALF);
  return QCU_SUCCESS;
}

int qcuContextHalfOperator(qcu_context ctx, int nrhs) {
  clear_error();
  const int st = ctx_check(ctx);
  if (st != QCU_SUCCESS) return -st;
  if (nrhs < 1) {
    set_error(QCU_ERR_INVALID_ARG, "nrhs must be positive");
    return -QCU_ERR_INVALID_ARG;
  }
  return ctx_op(ctx, PREC_HALF, nrhs) == OP_HALF ? 0 : 1;
}

long long qcuContextDeviceBytes(qcu_context ctx) {
  if (!ctx) return 0;
  long long n = ctx->gauge64.bytes + ctx->gauge32.bytes + ctx->gauge16.bytes + ctx->gauge18.bytes;
  n += qcu_engine_device_bytes(ctx);
  n += ctx->clover.A64.bytes + ctx->clover.Ainv64.bytes + ctx->clover.Ainv32.bytes + ctx->clover.Ainv16.bytes +
       ctx->clover.F64.bytes;
  n += ctx->red.partial.bytes + ctx->lin.data.bytes + ctx->lout.data.bytes + ctx->ltmp.data.bytes +
       ctx->ltmp2.data.bytes + ctx->lx.data.bytes + ctx->stage_in.bytes + ctx->stage_out.bytes;
  return n;
}

long long qcuContextLaunchCount(qcu_context ctx) { return ctx ? ctx->launches : 0; }

void qcuDebugFailAllocAfter(long long n) { set_alloc_fail_after(n); }
void qcuDebugSetPairStage(int stage) { set_pair_stage_override(stage); }

int qcuLoadGauge(qcu_context ctx, const void* gauge) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (!gauge) {
    set_error(QCU_ERR_INVALID_ARG, "null gauge");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK(ingest_gauge(ctx, gauge));
  ctx->legacy_gauge_src = nullptr;
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}

int qcuGenerateGauge(qcu_context ctx, unsigned long long seed, double eps) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (ctx->g.tdd) return dd_generate_gauge(ctx, seed, eps);
  size_t aos_bytes = (size_t)8 * ctx->g.Vh * 9 * 16;
  DevBuf tmp;
  QCU_CHECK(tmp.ensure(aos_bytes, ctx->stream));
  QCU_CHECK_CUDA(launch_gauge_random(ctx->g, seed, eps, tmp.p, ctx->stream));
  ctx->launches++;
  QCU_CHECK(ingest_gauge(ctx, tmp.p));
  ctx->legacy_gauge_src = nullptr;
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}

int qcuExportGauge(qcu_context ctx, void* out);  // below (needs a kernel-free path)

int qcuGenerateSpinor(qcu_context ctx, void* out, int nrhs, unsigned long long seed) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (!out || nrhs < 1) {
    set_error(QCU_ERR_INVALID_ARG, "bad spinor arguments");
    return QCU_ERR_INVALID_ARG;
  }
  size_t per = (size_t)2 * ctx->g.Vh;  // sites of one full spinor
  bool dev = is_device_ptr(out);
  void* dst = out;
  if (!dev) {
    QCU_CHECK(ctx->stage_out.ensure(per * 192 * nrhs, ctx->stream));
    dst = ctx->stage_out.p;
  }
  for (int r = 0; r < nrhs; r++) {
    char* d = static_cast<char*>(dst) + per * 192 * r;
    if (ctx->g.tdd)  // the slab's part of the global field's spinor
      QCU_CHECK_CUDA(launch_spinor_random_slab(ctx->g, ctx->Lt_global, ctx->t0, seed + r, d, ctx->stream));
    else
      QCU_CHECK_CUDA(launch_spinor_random(per, seed + r, d, ctx->stream));
    ctx->launches++;
  }
  if (!dev) QCU_CHECK_CUDA(cudaMemcpyAsync(out, dst, per * 192 * nrhs, cudaMemcpyDeviceToHost, ctx->stream));
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}

int qcuDslash(qcu_context ctx, void* out, const void* in, int parity, int dagger, double bc_t) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (!out || !in || (parity != 0 && parity != 1)) {
    set_error(QCU_ERR_INVALID_ARG, "bad dslash arguments");
    return QCU_ERR_INVALID_ARG;
  }
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  QCU_CHECK(spinor_to_internal(ctx, in, ctx->lin, 1));
  QCU_CHECK(ctx->lout.alloc(PREC_DOUBLE, ctx->g.Vh_pad, 1, 1, ctx->stream));
  DslashArgs a = base_args(ctx, PREC_DOUBLE);
  a.parity = parity;
  a.in = ctx->lin.cview(0);
  a.out = ctx->lout.view(0);
  a.bc_t = bc_t;
  QCU_CHECK(run_dslash(ctx, PREC_DOUBLE, dagger != 0, 0, a));
  QCU_CHECK(spinor_from_internal(ctx, ctx->lout, out, 1));
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}

int qcuApplyClover(qcu_context ctx, void* out, const void* in, double csw_eff, int inverse) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (!out || !in) {
    set_error(QCU_ERR_INVALID_ARG, "null spinor");
    return QCU_ERR_INVALID_ARG;
  }
  int slot;
  QCU_CHECK(ctx_clover_slot(ctx, csw_eff, &slot));
  QCU_CHECK(spinor_to_internal(ctx, in, ctx->lin, 2));
  QCU_CHECK(ctx->lout.alloc(PREC_DOUBLE, ctx->g.Vh_pad, 1, 2, ctx->stream));
  QCU_CHECK(clover_both(ctx, ctx->lin, ctx->lout, inverse != 0, slot));
  QCU_CHECK(spinor_from_internal(ctx, ctx->lout, out, 2));
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}

int qcuApplyOperator(qcu_context ctx, void* out, const void* in, double kappa, double csw, double bc_t, int dagger) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (!out || !in) {
    set_error(QCU_ERR_INVALID_ARG, "null spinor");
    return QCU_ERR_INVALID_ARG;
  }
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  int slot = -1;
  if (csw != 0.0) QCU_CHECK(ctx_clover_slot(ctx, kappa * csw, &slot));
  QCU_CHECK(spinor_to_internal(ctx, in, ctx->lin, 2));
  QCU_CHECK(ctx->lout.alloc(PREC_DOUBLE, ctx->g.Vh_pad, 1, 2, ctx->stream));
  for (int p = 0; p < 2; p++) {
    DslashArgs a = base_args(ctx, PREC_DOUBLE);
    a.parity = p;
    a.in = ctx->lin.cview(1 - p);
    a.out = ctx->lout.view(p);
    a.x = ctx->lin.cview(p);
    a.coef0 = -kappa;
    a.bc_t = bc_t;
    int epi = EPI_XPAY;
    if (slot >= 0) {
      epi |= EPI_CX;
      a.clover = clover_at(ctx, PREC_DOUBLE, false, slot);
    }
    QCU_CHECK(run_dslash(ctx, PREC_DOUBLE, dagger != 0, epi, a));
  }
  QCU_CHECK(spinor_from_internal(ctx, ctx->lout, out, 2));
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}

// ---------------- reference interface ----------------

void initGridSize(QcuGrid_t* grid, QcuParam* p_param, void* gauge, void* fermion_in, void* fermion_out) {
  (void)fermion_in;
  (void)fermion_out;
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  clear_error();
  if (!grid || !p_param) {
    set_error(QCU_ERR_INVALID_ARG, "null grid or param");
    return;
  }
  for (int i = 0; i < 4; i++)
    if (grid->grid_size[i] != 1) {
      set_error(QCU_ERR_UNSUPPORTED, "only the process grid {1,1,1,1} is supported (one GPU)");
      return;
    }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    dev = 0;
  }
  if (g_legacy) {
    qcuContextDestroy(g_legacy);
    g_legacy = nullptr;
  }
  qcu_context ctx = nullptr;
  if (qcuContextCreate(&ctx, p_param->lattice_size, dev) != QCU_SUCCESS) return;
  g_legacy = ctx;
  g_legacy->legacy_gauge_src = nullptr;
  (void)gauge;  // read lazily by the first call that needs it
}

void loadQcuGauge(void* gauge, QcuParam* param) {
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  if (legacy_begin(param, nullptr, &ctx) != QCU_SUCCESS) return;
  if (!gauge) {
    set_error(QCU_ERR_INVALID_ARG, "null gauge");
    return;
  }
  int st = ingest_gauge(ctx, gauge);
  if (st == QCU_SUCCESS) ctx->legacy_gauge_src = gauge;
  legacy_finish(ctx, st);
}

void dslashQcu(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int parity) {
  NvtxRange nv("dslashQcu");
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  if (legacy_begin(param, gauge, &ctx) != QCU_SUCCESS) return;
  int st = qcuDslash(ctx, fermion_out, fermion_in, parity, 0, 1.0);
  legacy_finish(ctx, st);
}

static int legacy_full(qcu_context ctx, void* out, void* in, int kind, int dag) {
  int slot;
  QCU_CHECK(ctx_clover_slot(ctx, 1.0, &slot));
  QCU_CHECK(spinor_to_internal(ctx, in, ctx->lin, 2));
  QCU_CHECK(ctx->lout.alloc(PREC_DOUBLE, ctx->g.Vh_pad, 1, 2, ctx->stream));
  QCU_CHECK(full_round(ctx, kind, ctx->lin, ctx->lout, dag != 0, slot));
  QCU_CHECK(spinor_from_internal(ctx, ctx->lout, out, 2));
  return QCU_SUCCESS;
}

void fullDslashQcu(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int dagger_flag) {
  NvtxRange nv("fullDslashQcu");
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  if (legacy_begin(param, gauge, &ctx) != QCU_SUCCESS) return;
  if (!fermion_out || !fermion_in) {
    set_error(QCU_ERR_INVALID_ARG, "null spinor");
    return;
  }
  legacy_finish(ctx, legacy_full(ctx, fermion_out, fermion_in, ROUND_FULL, dagger_flag));
}

static int legacy_clover_inplace(qcu_context ctx, void* out, bool inverse) {
  int slot;
  QCU_CHECK(ctx_clover_slot(ctx, 1.0, &slot));
  QCU_CHECK(spinor_to_internal(ctx, out, ctx->lin, 2));
  QCU_CHECK(ctx->lout.alloc(PREC_DOUBLE, ctx->g.Vh_pad, 1, 2, ctx->stream));
  QCU_CHECK(clover_both(ctx, ctx->lin, ctx->lout, inverse, slot));
  QCU_CHECK(spinor_from_internal(ctx, ctx->lout, out, 2));
  return QCU_SUCCESS;
}

void invertCloverDslash(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag) {
  (void)fermion_in;
  (void)invert_flag;
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  if (legacy_begin(param, gauge, &ctx) != QCU_SUCCESS) return;
  if (!fermion_out) {
    set_error(QCU_ERR_INVALID_ARG, "null spinor");
    return;
  }
  legacy_finish(ctx, legacy_clover_inplace(ctx, fermion_out, true));
}

int qcuPreCloverDslash(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag) {
  (void)fermion_in;
  (void)invert_flag;
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  QCU_CHECK(legacy_begin(param, gauge, &ctx));
  if (!fermion_out) {
    set_error(QCU_ERR_INVALID_ARG, "null spinor");
    return QCU_ERR_INVALID_ARG;
  }
  return legacy_finish(ctx, legacy_clover_inplace(ctx, fermion_out, false));
}

int qcuCloverDslashOneRound(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag) {
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  QCU_CHECK(legacy_begin(param, gauge, &ctx));
  return legacy_finish(ctx, legacy_full(ctx, fermion_out, fermion_in, ROUND_CLOVER_HOP, invert_flag));
}

int qcuFullCloverDslashOneRound(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag) {
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  QCU_CHECK(legacy_begin(param, gauge, &ctx));
  return legacy_finish(ctx, legacy_full(ctx, fermion_out, fermion_in, ROUND_FULL, invert_flag));
}

int qcuNewFullCloverDslashOneRound(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag) {
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  QCU_CHECK(legacy_begin(param, gauge, &ctx));
  return legacy_finish(ctx, legacy_full(ctx, fermion_out, fermion_in, ROUND_NEWFULL, invert_flag));
}

int qcuMmVOneRound(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, void* temp) {
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  QCU_CHECK(legacy_begin(param, gauge, &ctx));
  int slot;
  QCU_CHECK(ctx_clover_slot(ctx, 1.0, &slot));
  QCU_CHECK(spinor_to_internal(ctx, fermion_in, ctx->lin, 2));
  QCU_CHECK(ctx->ltmp.alloc(PREC_DOUBLE, ctx->g.Vh_pad, 1, 2, ctx->stream));
  QCU_CHECK(ctx->lout.alloc(PREC_DOUBLE, ctx->g.Vh_pad, 1, 2, ctx->stream));
  QCU_CHECK(full_round(ctx, ROUND_NEWFULL, ctx->lin, ctx->ltmp, false, slot));
  QCU_CHECK(full_round(ctx, ROUND_NEWFULL, ctx->ltmp, ctx->lout, true, slot));
  if (temp) QCU_CHECK(spinor_from_internal(ctx, ctx->ltmp, temp, 2));
  QCU_CHECK(spinor_from_internal(ctx, ctx->lout, fermion_out, 2));
  return legacy_finish(ctx, QCU_SUCCESS);
}

// The reference's C++ entry points, under their C++ symbol names, so a binary
// linked against the reference resolves them here (names as the reference's
// compiler emits them for include/qcu_clover_dslash.cuh:15-25).
void qcu_cxx_invertCloverDslash(void* o, void* i, void* g, QcuParam* p, int f) __asm__("_Z18invertCloverDslashPvS_S_P10QcuParam_si");
void qcu_cxx_invertCloverDslash(void* o, void* i, void* g, QcuParam* p, int f) { invertCloverDslash(o, i, g, p, f); }
void qcu_cxx_preCloverDslash(void* o, void* i, void* g, QcuParam* p, int f) __asm__("_Z15preCloverDslashPvS_S_P10QcuParam_si");
void qcu_cxx_preCloverDslash(void* o, void* i, void* g, QcuParam* p, int f) { qcuPreCloverDslash(o, i, g, p, f); }
void qcu_cxx_cloverDslashOneRound(void* o, void* i, void* g, QcuParam* p, int f) __asm__("_Z20cloverDslashOneRoundPvS_S_P10QcuParam_si");
void qcu_cxx_cloverDslashOneRound(void* o, void* i, void* g, QcuParam* p, int f) { qcuCloverDslashOneRound(o, i, g, p, f); }
void qcu_cxx_fullCloverDslashOneRound(void* o, void* i, void* g, QcuParam* p, int f) __asm__("_Z24fullCloverDslashOneRoundPvS_S_P10QcuParam_si");
void qcu_cxx_fullCloverDslashOneRound(void* o, void* i, void* g, QcuParam* p, int f) { qcuFullCloverDslashOneRound(o, i, g, p, f); }
void qcu_cxx_newFullCloverDslashOneRound(void* o, void* i, void* g, QcuParam* p, int f) __asm__("_Z27newFullCloverDslashOneRoundPvS_S_P10QcuParam_si");
void qcu_cxx_newFullCloverDslashOneRound(void* o, void* i, void* g, QcuParam* p, int f) { qcuNewFullCloverDslashOneRound(o, i, g, p, f); }
void qcu_cxx_MmV_one_round(void* o, void* i, void* g, QcuParam* p, void* t) __asm__("_Z13MmV_one_roundPvS_S_P10QcuParam_sS_");
void qcu_cxx_MmV_one_round(void* o, void* i, void* g, QcuParam* p, void* t) { qcuMmVOneRound(o, i, g, p, t); }

}  // extern "C"

// ---------------------------------------------------------------------------
// the reference CG flow, src/cg_inverter.cu:181-369
// ---------------------------------------------------------------------------
static int ref_cg(qcu_context ctx, void* b_vec, void* x_vec, int* iters_out, bool* conv_out) {
  const Geom& g = ctx->g;
  int slot;
  QCU_CHECK(ctx_clover_slot(ctx, 1.0, &slot));
  Field b, x, r, r2, p, ap, tmp, nb;
  cudaStream_t st = ctx->stream;
  QCU_CHECK(spinor_to_internal(ctx, b_vec, b, 2));
  for (Field* f : {&x, &r, &r2, &p, &ap, &tmp, &nb}) QCU_CHECK(f->alloc(PREC_DOUBLE, g.Vh_pad, 1, 2, st));
  const int n = 2 * g.Vh_pad;
  QCU_CHECK(ctx->red.ensure(g, 1, st, ctx->shape1.Sb));
  ReduceArgs red = ctx->red.args();
  double* h = ctx->red.host.as<double>();
  auto dot = [&](const Field& u, const Field& v, double out[2]) -> int {
    QCU_CHECK_CUDA(launch_cdot(PREC_DOUBLE, n, 1, u.cview(0), v.cview(0), nullptr, red, ctx->shape1, st));
    ctx->launches++;
    QCU_CHECK_CUDA(cudaMemcpyAsync(h, ctx->red.result.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    QCU_CHECK_CUDA(cudaStreamSynchronize(st));
    out[0] = h[0];
    out[1] = h[1];
    return QCU_SUCCESS;
  };
  // tmp = A^-1 b ; nb = (1 - A^-1 D^dag) tmp ; x = 0 ; r = nb ; p = r
  QCU_CHECK(clover_both(ctx, b, tmp, true, slot));
  QCU_CHECK(full_round(ctx, ROUND_NEWFULL, tmp, nb, true, slot));
  QCU_CHECK_CUDA(cudaMemcpyAsync(r.data.p, nb.data.p, r.data.bytes, cudaMemcpyDeviceToDevice, st));
  QCU_CHECK_CUDA(cudaMemcpyAsync(p.data.p, nb.data.p, p.data.bytes, cudaMemcpyDeviceToDevice, st));
  double num[2];
  QCU_CHECK(dot(r, r, num));
  const long long maxit = (long long)2 * g.Vh;  // V, src/cg_inverter.cu:268
  int it = 0;
  bool conv = hypot(num[0], num[1]) < 1e-23;
  while (!conv && it < maxit) {
    QCU_CHECK(full_round(ctx, ROUND_NEWFULL, p, tmp, false, slot));
    QCU_CHECK(full_round(ctx, ROUND_NEWFULL, tmp, ap, true, slot));
    double den[2];
    QCU_CHECK(dot(p, ap, den));
    double dd = den[0] * den[0] + den[1] * den[1];
    double2 alpha = make_double2((num[0] * den[0] + num[1] * den[1]) / dd, (num[1] * den[0] - num[0] * den[1]) / dd);
    QCU_CHECK_CUDA(launch_ref_xr(n, x.view(0), p.cview(0), r.cview(0), ap.cview(0), r2.view(0), alpha, red, ctx->shape1, st));
    ctx->launches++;
    QCU_CHECK_CUDA(cudaMemcpyAsync(h, ctx->red.result.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    QCU_CHECK_CUDA(cudaStreamSynchronize(st));
    double rr2[2] = {h[0], h[1]};
    it++;
    if (hypot(num[0], num[1]) < 1e-23) {  // the residual from before the update (src/cg_inverter.cu:225)
      conv = true;
      break;
    }
    double nn = num[0] * num[0] + num[1] * num[1];
    double2 beta = make_double2((rr2[0] * num[0] + rr2[1] * num[1]) / nn, (rr2[1] * num[0] - rr2[0] * num[1]) / nn);
    QCU_CHECK_CUDA(launch_ref_p(n, p.view(0), r2.cview(0), beta, ctx->shape1, st));
    ctx->launches++;
    std::swap(r.data.p, r2.data.p);
    num[0] = rr2[0];
    num[1] = rr2[1];
    if (!isfinite(num[0])) break;
  }
  QCU_CHECK(spinor_from_internal(ctx, x, x_vec, 2));
  QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  *iters_out = it;
  *conv_out = conv;
  return QCU_SUCCESS;
}

extern "C" {

void cg_inverter(void* b_vector, void* x_vector, void* gauge, QcuParam* param) {
  NvtxRange nv("cg_inverter");
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  if (legacy_begin(param, gauge, &ctx) != QCU_SUCCESS) return;
  if (!b_vector || !x_vector) {
    set_error(QCU_ERR_INVALID_ARG, "null spinor");
    return;
  }
  int it = 0;
  bool conv = false;
  int st = ref_cg(ctx, b_vector, x_vector, &it, &conv);
  if (st != QCU_SUCCESS) return;
  // the reference reports on stdout (src/cg_inverter.cu:330, 342-349)
  if (!getenv("QCU_QUIET")) {
    if (conv && it > 0) printf("number of iteration %d\n", it);
    printf(conv ? "cg success!!!\n" : "cg_failed!!!\n");
  }
  if (!conv) set_error(QCU_ERR_NOT_CONVERGED, "reference CG flow did not reach |<r,r>| < 1e-23");
}

// Extended-API variant of the reference flow: iterations and convergence out.
int qcuCgInverterRef(void* b_vector, void* x_vector, void* gauge, QcuParam* param, int* iterations, int* converged) {
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  qcu_context ctx;
  QCU_CHECK(legacy_begin(param, gauge, &ctx));
  int it = 0;
  bool conv = false;
  QCU_CHECK(ref_cg(ctx, b_vector, x_vector, &it, &conv));
  if (iterations) *iterations = it;
  if (converged) *converged = conv ? 1 : 0;
  return conv ? QCU_SUCCESS : QCU_ERR_NOT_CONVERGED;
}

qcu_context qcuLegacyContext(void) { return g_legacy; }

}  // extern "C"
