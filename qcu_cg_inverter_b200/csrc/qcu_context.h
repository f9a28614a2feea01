// Host-side state of the library: device buffers, the resident gauge field,
// the bank of factored clover fields, reduction scratch and the error
// channel. Replaces the reference's process globals (static clover and
// inverse, src/qcu_clover_dslash.cu:564-568; qcu_gauge, src/dslash.cu:26;
// mpi_comm, src/qcu_communicator.cu:1031) by an explicit context.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/qcu_b200.h"
#include "qcu_cg_state.cuh"
#include "qcu_common.cuh"
#include "qcu_fields.cuh"
#include "qcu_kernels.cuh"

namespace qcu {

// NVTX range for the scope of a C entry point or a solver phase (visible in
// nsys / ncu timelines; costs a few ns when no tool is attached)
struct NvtxRange {
  explicit NvtxRange(const char* name);
  ~NvtxRange();
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// ---------------- errors ----------------
void set_error(int code, const std::string& msg);
void clear_error();
int last_error();

// converts a CUDA error into a status (and records it)
int cuda_status(cudaError_t e, const char* what);

#define QCU_CHECK_CUDA(expr)                                       \
  do {                                                             \
    cudaError_t _e = (expr);                                       \
    if (_e != cudaSuccess) return ::qcu::cuda_status(_e, #expr);   \
  } while (0)
#define QCU_CHECK(expr)                \
  do {                                 \
    int _s = (expr);                   \
    if (_s != QCU_SUCCESS) return _s;  \
  } while (0)

// ---------------- device memory ----------------
// Test hook: after `n` more successful allocations the next one fails
// (negative n = never). Used by the host-side fault tests.
void set_alloc_fail_after(long long n);
cudaError_t dev_alloc(void** p, size_t bytes);

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  // (re)allocates to at least `n` bytes, zero-filled
  int ensure(size_t n, cudaStream_t st);
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() { release(); }
  int ensure(size_t n);
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// ---------------- spinor fields ----------------
struct Field {
  int prec = PREC_DOUBLE;
  int nrhs = 0;
  int nsites = 0;  // sites per parity block (Vh_pad)
  int nparity = 1;
  DevBuf data, norm;
  int alloc(int prec_, int nsites_, int nrhs_, int nparity_, cudaStream_t st);
  SpinorView view(int parity = 0) const;
  CSpinorView cview(int parity = 0) const { return CSpinorView(view(parity)); }
  size_t parity_bytes() const { return spinor_field_bytes(prec, nsites, nrhs); }
  size_t parity_norm_bytes() const { return spinor_norm_bytes(prec, nsites, nrhs); }
};

// ---------------- clover bank ----------------
// Factored clover fields for several values of csw_eff = kappa*c_sw, each
// slot holding A (FP64) and A^-1 (FP64, single, 16-bit), all slots of one
// precision in one allocation so that a kernel can address slot k as
// base + k*stride (one right-hand side per kappa in a batch).
struct CloverBank {
  int capacity = 0;
  size_t b64 = 0, b32 = 0, b16 = 0;
  DevBuf A64, Ainv64, Ainv32, Ainv16;
  DevBuf F64;                     // the kappa-independent field term of the current links
  long long F_version = -1;       // gauge_version F64 belongs to
  std::vector<double> csw;       // csw_eff of each slot (NaN = free)
  std::vector<long long> stamp;  // last use, for eviction
  std::vector<int> pinned;       // slots used by the batch being prepared
};

struct Scratch {
  DevBuf partial, ticket, result, partial2, group_ticket;
  PinnedBuf host;
  size_t partial_doubles = 0;
  // min_sb: the fewest site lanes per block of any launch that reduces
  int ensure(const Geom& g, int nrhs, cudaStream_t st, int min_sb);
  ReduceArgs args(void* state = nullptr) const {
    return ReduceArgs{partial.as<double>(), ticket.as<unsigned>(), result.as<double>(), state,
                      partial2.as<double>(), group_ticket.as<unsigned>()};
  }
};

class Engine;  // engine.cu

}  // namespace qcu

struct qcu_context_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  int L[4] = {0, 0, 0, 0};
  qcu::Geom g{};
  // resident gauge field (internal layout): 12-real double/single/16-bit and
  // 18-real single (the fast 16-bit operator's links)
  qcu::DevBuf gauge64, gauge32, gauge16, gauge18;
  // operator variant behind QCU_PREC_HALF: OP_HALF_FAST, OP_HALF, or -1 =
  // chosen per solve (ctx_op)
  int half_op = -1;
  bool gauge_loaded = false;
  long long gauge_version = 0;
  const void* legacy_gauge_src = nullptr;  // AoS pointer last ingested by the legacy API
  qcu::CloverBank clover;
  long long clock = 0;
  qcu::Scratch red;
  qcu::LaunchShape shape1{1, 128};  // single-RHS stencil/BLAS shape
  bool shape_set = false;           // shape1 set by qcuContextSetShape
  // scratch fields for the legacy and operator entry points
  qcu::Field lin, lout, ltmp, ltmp2, lx;
  qcu::DevBuf stage_in, stage_out;  // device staging of host arguments
  qcu::DevBuf status;               // clover build status counters
  qcu::Engine* engine = nullptr;  // batch engine of qcuInvert; owned, freed by qcuContextDestroy (engine.cu)
  std::map<std::pair<int, int>, qcu::LaunchShape> tuned;  // (precision, nrhs) -> block shape (tune.cu)
  bool tune_cache_loaded = false;
  long long clover_gen = 0;  // bumped whenever the clover bank moves
  long long launches = 0;
  // t-slab of a decomposed lattice (comm.cu): the communicator, the global
  // time extent and this slab's first global slice, and the extended slab
  // (two more slices on each side, periodic) that ingests the gauge field and
  // builds the clover term
  qcu_comm comm = nullptr;
  int Lt_global = 0, t0 = 0;
  qcu_context ext = nullptr;
  cudaStream_t dd_stream = nullptr;  // the halo exchange, beside the interior stencil
  cudaEvent_t dd_ev[2] = {nullptr, nullptr};
  ~qcu_context_s();
};

namespace qcu {

// context helpers (api.cu). `op` arguments are OpVariant values (PREC_*
// values are the matching uniform variants).
int ctx_check(qcu_context ctx);
// Builds on demand. wait = false enqueues the build without reading back its
// pivot check (a singular block then shows up as a breakdown of the solve).
int ctx_clover_slot(qcu_context ctx, double csw_eff, int* slot, bool wait = true);
// Replaces the context's stream by one with this scheduling priority
// (cudaDeviceGetStreamPriorityRange); only while no work is queued on it.
int ctx_set_stream_priority(qcu_context ctx, int priority);
int ctx_clover_reserve(qcu_context ctx, int nslots);
const void* ctx_clover_ptr(qcu_context ctx, int op, bool inverse);
size_t ctx_clover_stride(qcu_context ctx, int op);
const void* ctx_gauge(qcu_context ctx, int op);
// the operator variant that serves spinor precision `prec`
// Half volumes from which single-RHS 16-bit solves keep links and clover in
// 16-bit (OP_HALF) by default. Measured on B200: at 32^3x64 (fields far beyond
// L2) the fused CG stencil takes 162 instead of 208 us and the solve 28.8
// instead of 35.8 ms; at 16^3x32 (the FP32 fields, 80 MB, fit in L2) the FP32
// links are faster per launch (14.4 vs 16.4 us) and the solves are even.
constexpr int kCompactMinVh = 131072;
// the operator variant that serves spinor precision `prec` for a solve or
// launch of nrhs right-hand sides
inline int ctx_op(qcu_context ctx, int prec, int nrhs) {
  if (prec != PREC_HALF) return prec;
  if (ctx->half_op >= 0) return ctx->half_op;
  return (nrhs == 1 && ctx->g.Vh_pad >= kCompactMinVh) ? (int)OP_HALF : (int)OP_HALF_FAST;
}

// launch shapes (tune.cu)
LaunchShape ctx_shape(qcu_context ctx, int prec, int nrhs);
bool ctx_is_tuned(qcu_context ctx, int prec, int nrhs);
int ctx_autotune(qcu_context ctx, int prec, int nrhs, double* best_ms);

// staging of user pointers that may live on the host
bool is_device_ptr(const void* p);
// device memory of `device` (or managed memory)
bool is_device_ptr_on(const void* p, int device);
// qcuDslashNoAlloc's set-up on the current device (noalloc.cu): the scratch
// array's device address and the code of the kernels it launches
int noalloc_prepare(int device);
cudaError_t preload_spinor_io_f64();

// t-slab decomposition (comm.cu): ghost slices of a spinor view of precision
// `prec` from the neighbouring ranks, and global sums of n doubles in place
// (both no-ops on a context that is not a slab)
int dd_exchange(qcu_context ctx, const CSpinorView& v, int prec, cudaStream_t st);
int dd_sum(qcu_context ctx, double* values, int n, cudaStream_t st);
// One stencil on a slab with the exchange of its input's faces overlapped:
// `launch` enqueues a piece of the stencil (a over a site range) on st; the
// interior slices run while the faces travel on the context's exchange
// stream, then the first and last slices. The pieces share a's reduction.
int dd_stencil(qcu_context ctx, const DslashArgs& a, int prec, LaunchShape sh, cudaStream_t st,
               const std::function<cudaError_t(const DslashArgs&)>& launch);
// copies the slab's part of the extended slab's clover slot into its own slot
int dd_clover_from_ext(qcu_context ctx, int ext_slot, int slot);
// the finishing functor `fin` (FinId) applied to reduced totals, as the
// reduction's last block would have (solver.cu)
cudaError_t launch_fin(int fin, const ReduceArgs& red, int nrhs, cudaStream_t st);
bool dd_graphs_ok(qcu_context ctx);

// kernel launchers (defined in the .cu files)
cudaError_t launch_gauge_ingest(const Geom& g, const void* aos, void* d64, void* d32, void* d16, void* d18,
                                cudaStream_t st);
// count AoS spinors (RHS r at aos + r*aos_stride complex) <-> RHS columns
// r0 .. r0+count-1 of an internal field
cudaError_t launch_spinor_in(int prec, const Geom& g, int count, const void* aos, size_t aos_stride, SpinorView dst,
                             cudaStream_t st, int r0 = 0);
cudaError_t launch_spinor_out(int prec, const Geom& g, int count, CSpinorView src, void* aos, size_t aos_stride,
                              cudaStream_t st, int r0 = 0);
cudaError_t launch_gauge_random(const Geom& g, uint64_t seed, double eps, void* aos, cudaStream_t st);
cudaError_t launch_spinor_random(size_t nsites, uint64_t seed, void* aos, cudaStream_t st);
// the same seeded fields restricted to a t-slab of a global lattice of time
// extent lt_glob: the links of slices t_first .. t_first + g.Lt - 1 (modulo
// lt_glob) and one full spinor of the slab starting at slice t0
cudaError_t launch_gauge_random_slab(const Geom& g, int lt_glob, int t_first, uint64_t seed, double eps, void* aos,
                                     cudaStream_t st);
cudaError_t launch_spinor_random_slab(const Geom& g, int lt_glob, int t0, uint64_t seed, void* aos, cudaStream_t st);
int ingest_gauge(qcu_context ctx, const void* gauge);
// slab contexts (comm.cu): the gauge field of the slab (local AoS), or the
// seeded field of the global lattice restricted to the slab
int dd_ingest_gauge(qcu_context ctx, const void* gauge);
int dd_generate_gauge(qcu_context ctx, uint64_t seed, double eps);
// A = 1 + csw_eff F and its inverse into the given fields; F (the
// kappa-independent field term, one packed FP64 field) is built from the links
// first unless F_ready
cudaError_t launch_clover_build(const Geom& g, const void* gauge64, double csw_eff, void* A64, void* Ainv64,
                                void* Ainv32, void* Ainv16, int* status, cudaStream_t stream, void* F64, bool F_ready);
cudaError_t launch_clover_apply(int prec, const Geom& g, int parity, int nrhs, CSpinorView in, SpinorView out,
                                const void* clov, size_t clov_stride, const int* clov_idx, const int* active,
                                const ReduceArgs* red, LaunchShape sh, cudaStream_t stream);
cudaError_t launch_cg_p(int pa, int ps, int nsites, int nrhs, SpinorView p, CSpinorView r, const double* beta,
                        const int* active, LaunchShape sh, cudaStream_t st);
cudaError_t launch_convert(int pd, int psrc, int nsites, int nrhs, SpinorView dst, CSpinorView src, const int* active,
                           const ReduceArgs* red, LaunchShape sh, cudaStream_t st);
cudaError_t launch_accumulate(int pl, int nsites, int nrhs, SpinorView xhi, SpinorView xlo, const int* active,
                              LaunchShape sh, cudaStream_t st);
cudaError_t launch_zero(int prec, int nsites, int nrhs, SpinorView f, const int* active, LaunchShape sh,
                        cudaStream_t st);
cudaError_t launch_accumulate_res(int pl, int nsites, int nrhs, SpinorView xhi, SpinorView xlo, CSpinorView b,
                                  SpinorView d, const int* active, LaunchShape sh, cudaStream_t st);
// |A r|^2 per RHS (into red) and u = A^-1 r in one pass from the FP64 r, FP64
// clover fields; u in precision pu, and for pu other than FP64 also r rounded
// to pu into rs. fin: FIN_NONE, or FIN_REL_CONT (red.state the CG state) to
// mark the RHS that go on after the reliable update.
cudaError_t launch_clover_res(int pu, const Geom& g, int parity, int nrhs, CSpinorView r, SpinorView u, SpinorView rs,
                              const void* A, const void* Ainv, size_t clov_stride, const int* clov_idx,
                              const int* active, const ReduceArgs& red, LaunchShape sh, cudaStream_t stream,
                              int fin = 0);
cudaError_t launch_residual(int nsites, int nrhs, SpinorView r, CSpinorView b, CSpinorView z, const int* active,
                            const ReduceArgs& red, LaunchShape sh, cudaStream_t st);
cudaError_t launch_cdot(int prec, int nsites, int nrhs, CSpinorView x, CSpinorView y, const int* active,
                        const ReduceArgs& red, LaunchShape sh, cudaStream_t st);
cudaError_t launch_ref_xr(int nsites, SpinorView x, CSpinorView p, CSpinorView r, CSpinorView ap, SpinorView r2,
                          double2 a, const ReduceArgs& red, LaunchShape sh, cudaStream_t st);
cudaError_t launch_ref_p(int nsites, SpinorView p, CSpinorView r2, double2 b, LaunchShape sh, cudaStream_t st);

}  // namespace qcu
