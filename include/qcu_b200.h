/*
 * qcu_b200.h - extended C interface of the B200 Wilson-clover solver.
 *
 * Everything here returns a status code (QCU_SUCCESS = 0) instead of exiting.
 * Two groups of entry points:
 *
 *  1. The reference's operator compositions, which it declares with C++
 *     linkage in cg_inverter/include/qcu_clover_dslash.cuh:15-25 and calls
 *     from its CG (src/qcu_clover_dslash.cu:920-1049). They use the context
 *     created by initGridSize() and keep the reference's argument meaning.
 *     The library also exports them under the reference's C++ symbol names,
 *     so a binary built against the reference resolves them too.
 *
 *  2. New, context-based entry points for the physical operator
 *       M = A - kappa*D,   A = 1 + kappa*c_sw*T
 *     (T the reference's clover term, i.e. A = 1 - (kappa c_sw/2) sigma.F),
 *     with an antiperiodic-in-time option, the even-odd preconditioned
 *     mixed-precision CG with reliable updates, and batched multi-RHS /
 *     multi-kappa solves. The reference has no counterpart for these; its
 *     CG hard-codes kappa = kappa*c_sw = 1 and periodic boundaries.
 *
 * Field arguments are complex-double AoS spinors in the reference layout
 * (see qcu.h). Unless stated, pointers may be device or host memory: host
 * data is staged through device buffers inside the call.
 */
#ifndef QCU_B200_H
#define QCU_B200_H

#include "qcu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
  QCU_SUCCESS = 0,
  QCU_ERR_INVALID_ARG = 1,
  QCU_ERR_CUDA = 2,
  QCU_ERR_NOT_CONVERGED = 3,
  QCU_ERR_OUT_OF_MEMORY = 4,
  QCU_ERR_TIMEOUT = 5,
  QCU_ERR_NOT_INITIALIZED = 6,
  QCU_ERR_UNSUPPORTED = 7,
  QCU_ERR_BREAKDOWN = 8,
  QCU_ERR_SINGULAR_CLOVER = 9,
  QCU_ERR_BUSY = 10
};

enum { QCU_PREC_DOUBLE = 0, QCU_PREC_SINGLE = 1, QCU_PREC_HALF = 2 };

/* ---- 1. reference compositions (context from initGridSize) ---- */

/* cloverDslashOneRound (src/qcu_clover_dslash.cu:990-1009):
 * out_p = A_p^-1 D^(dag) in_{1-p} for both parities, full spinors. */
int qcuCloverDslashOneRound(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag);
/* fullCloverDslashOneRound (src/qcu_clover_dslash.cu:948-987): out = (A - D^(dag)) in. */
int qcuFullCloverDslashOneRound(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag);
/* newFullCloverDslashOneRound (src/qcu_clover_dslash.cu:1013-1042): out = in - A^-1 D^(dag) in. */
int qcuNewFullCloverDslashOneRound(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag);
/* MmV_one_round (src/qcu_clover_dslash.cu:1044-1049):
 * out = (1 - A^-1 D^dag)(1 - A^-1 D) in; temp is a full-spinor work buffer. */
int qcuMmVOneRound(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, void* temp);
/* preCloverDslash (src/qcu_clover_dslash.cu:927-944): out <- A out in place
 * (fermion_in unused, as in the reference). */
int qcuPreCloverDslash(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag);
/* cg_inverter (src/cg_inverter.cu:260-369) with its outcome returned instead
 * of printed: iterations done and whether |<r,r>| < 1e-23 was reached. */
int qcuCgInverterRef(void* b_vector, void* x_vector, void* gauge, QcuParam* param, int* iterations, int* converged);

/* ---- 2. context-based API ---- */

typedef struct qcu_context_s* qcu_context;

typedef struct {
  double kappa;       /* hopping parameter (used when the kappas array is NULL) */
  double csw;         /* clover coefficient c_sw; 0 = plain Wilson */
  double bc_t;        /* +1 periodic, -1 antiperiodic in time */
  double tol;         /* target true residual |b - M x| / |b| of the full system */
  int maxiter;        /* cap on CG iterations per right-hand side */
  int precision;      /* inner (sloppy) precision: QCU_PREC_DOUBLE / _SINGLE / _HALF */
  double delta;       /* reliable-update factor: the true residual is recomputed in
                         FP64 when the iterated one fell by this factor (0 = default) */
  int use_graphs;     /* replay CUDA graphs of the inner iterations (1 = yes) */
  int autotune;       /* time the launch shapes for this (precision, nrhs) before the
                         first solve that uses them (1 = yes; see qcuAutotune) */
} qcu_solve_params;

typedef struct {
  int iterations;        /* CG iterations on Mhat^dag Mhat */
  int reliable_updates;  /* FP64 true-residual recomputations */
  int converged;         /* 1 when true_residual < tol */
  int status;            /* QCU_SUCCESS, QCU_ERR_NOT_CONVERGED or QCU_ERR_BREAKDOWN */
  double true_residual;  /* |b - M x|/|b| of the returned x, evaluated in FP64 */
  double kappa;
  double gbytes;         /* algorithmic bytes (1e9) the solve of this RHS moved: every stencil,
                            clover and BLAS pass of its iterations, reliable updates, admission
                            and retirement, each neighbour load counted, link and clover bytes
                            divided by the RHS that share one load */
  double seconds;        /* qcuInvert: device time of the whole call (shared by its RHS);
                            0 in request-server reports (see qcuServerQuery's latency) */
  double gbytes_per_s;   /* qcuInvert: the call's gbytes summed over its RHS / seconds; 0 otherwise */
} qcu_solve_report;

/* Fills params with the defaults: kappa 0.12, csw 0, bc_t -1, tol 1e-10,
 * maxiter 20000, precision half, delta 0 (= 2e-3 for 16-bit inner storage,
 * 1e-3 for single, 1e-12 for double), use_graphs 1, autotune 1. */
void qcuSolveParamsDefault(qcu_solve_params* params);

int qcuContextCreate(qcu_context* ctx, const int lattice[4], int device);
int qcuContextDestroy(qcu_context ctx);
/* Orders the context's own stream after the caller's stream (cudaStream_t):
 * work enqueued later by the context starts after what `stream` holds now.
 * The context's stream does not wait for any other stream by itself, so a
 * caller whose arguments come from kernels still pending on its own stream
 * calls this first (the Python binding does it for torch tensors, with
 * torch's current stream); the reference-interface entry points (qcu.h) order
 * themselves after the default stream, as the reference's calls ran on it. */
int qcuContextSetStream(qcu_context ctx, void* stream);
/* The context's own stream (cudaStream_t), for recording events around calls. */
void* qcuContextGetStream(qcu_context ctx);
/* Thread-block shape (RHS lanes x site lanes, 32..256 threads) of the
 * context's single-RHS kernels; the autotuner sets it from measurements. */
int qcuContextSetShape(qcu_context ctx, int rhs_lanes, int site_lanes);
/* Storage behind QCU_PREC_HALF: fast_links = 1 keeps 16-bit spinors with FP32
 * links (all 18 reals, nothing to decode or rebuild) and an FP32 clover
 * inverse; 0 keeps links (12 reals) and the clover inverse in 16-bit too
 * (about half the bytes per site); -1 (the default) picks per solve: 16-bit
 * links and clover for single-RHS solves on half volumes of 131072 sites or
 * more (where the fields exceed L2 and bytes bound the stencil), FP32 links
 * and clover otherwise (batched solves, whose link and clover loads serve
 * every RHS, and small lattices). */
int qcuContextSetHalfOperator(qcu_context ctx, int fast_links);
/* The storage a 16-bit solve of nrhs right-hand sides would use on this
 * context: 1 = FP32 links and clover, 0 = 16-bit (negative: an error code). */
int qcuContextHalfOperator(qcu_context ctx, int nrhs);
/* Device bytes the context holds now. */
long long qcuContextDeviceBytes(qcu_context ctx);

/* Gauge field in the reference AoS layout (device or host). */
int qcuLoadGauge(qcu_context ctx, const void* gauge);
/* Seeded synthetic SU(3) field U = exp(i eps H) on the device (the same
 * counter-based streams as the CPU oracle's generator). */
int qcuGenerateGauge(qcu_context ctx, unsigned long long seed, double eps);
/* Copies the resident gauge field out in the AoS layout (rows 3 rebuilt). */
int qcuExportGauge(qcu_context ctx, void* gauge_out);
/* nrhs seeded complex-Gaussian full spinors (AoS), RHS r seeded with seed + r. */
int qcuGenerateSpinor(qcu_context ctx, void* out, int nrhs, unsigned long long seed);

/* out (half spinor, parity) = D^(dag) in (half spinor, 1-parity), hopping
 * term with time boundary factor bc_t. */
int qcuDslash(qcu_context ctx, void* out, const void* in, int parity, int dagger, double bc_t);
/* Same result as qcuDslash, for callers that must not allocate device memory
 * during the call (a framework that already holds the GPU's memory in its own
 * pool, or a loop that cannot take cudaMalloc's implicit synchronisation).
 * No counterpart in the reference. Instead of the staging fields qcuDslash
 * allocates on first use, it uses a fixed 6 MiB scratch array compiled into
 * the library, so the lattice's half volume may be at most 16384 sites
 * (larger: QCU_ERR_INVALID_ARG). in/out must be device memory of the
 * context's GPU. Calls that overlap on the GPU share that array and race.
 * qcuContextCreate does the per-device set-up (the array's device address,
 * the code of the kernels the call launches), so the 6 MiB are held from the
 * first context on a device until the process exits; if that set-up failed
 * there, the first call retries it, so make one call before any stream
 * capture. The address is cached per device: after a cudaDeviceReset the
 * library must not be used again in that process. */
int qcuDslashNoAlloc(qcu_context ctx, void* out, const void* in, int parity, int dagger, double bc_t);
/* out = A in (inverse = 0) or A^-1 in (inverse = 1), full spinors, with
 * A = 1 + csw_eff*T (csw_eff = kappa*c_sw; 1 reproduces the reference). */
int qcuApplyClover(qcu_context ctx, void* out, const void* in, double csw_eff, int inverse);
/* out = M in or M^dag in, M = A(kappa*csw) - kappa*D, full spinors. */
int qcuApplyOperator(qcu_context ctx, void* out, const void* in, double kappa, double csw, double bc_t, int dagger);

/* Solves M x_r = b_r for nrhs right-hand sides stored back to back (full
 * spinors). kappas (length nrhs) may be NULL to use params->kappa for all.
 * All RHS are iterated together: each link load serves every RHS, and each
 * RHS keeps its own CG scalars and stops on its own. reports (length nrhs)
 * may be NULL. Returns QCU_ERR_NOT_CONVERGED if any RHS missed tol. */
int qcuInvert(qcu_context ctx, void* x, const void* b, int nrhs, const double* kappas,
              const qcu_solve_params* params, qcu_solve_report* reports);

/* ---- request server: continuous batching over resident configurations ----
 * No counterpart in the reference (its cg_inverter, src/cg_inverter.cu:260-369,
 * solves one right-hand side per call). Each registered gauge configuration
 * becomes resident on first use (gauge field, factored clover bank and a
 * batch of RHS columns) within a device-memory budget; idle configurations are
 * evicted to make room. A request (kappa, c_sw, nrhs sources) joins its
 * configuration's batch as soon as nrhs columns and a clover slot are free,
 * while the requests already there keep iterating; batches of different
 * configurations run on their own streams and overlap on the GPU. Sources and
 * solutions are full AoS spinors, host or device; host buffers should be
 * pinned (qcuHostAlloc), otherwise the copies block the loop. */
typedef struct qcu_server_s* qcu_server;

typedef struct {
  int precision;            /* inner precision (default QCU_PREC_HALF) */
  double tol;               /* true residual |b - M x|/|b| of every request (1e-10) */
  int maxiter;              /* per RHS (20000) */
  double bc_t;              /* time boundary factor (-1) */
  double delta;             /* reliable-update factor, 0 = default */
  int columns;              /* RHS columns per resident configuration (16) */
  int clover_slots;         /* factored clover fields per resident configuration (8) */
  long long device_budget;  /* device bytes for resident configurations (0 = 85% of free memory) */
  int autotune;             /* tune launch shapes when a configuration becomes resident (1) */
  int max_chunk;            /* most CG iterations between two admission points of a batch (8) */
} qcu_server_params;

void qcuServerParamsDefault(qcu_server_params* params);
int qcuServerCreate(qcu_server* server, int device, const qcu_server_params* params);
/* Waits for the device work of every resident configuration, then frees all. */
int qcuServerDestroy(qcu_server server);
/* Registers the seeded synthetic gauge configuration exp(i eps H) (the field
 * qcuGenerateGauge makes) on this lattice; *config_id names it in requests. */
int qcuServerAddConfig(qcu_server server, const int lattice[4], unsigned long long seed, double eps, int* config_id);
/* Makes a configuration resident now (otherwise done by its first request). */
int qcuServerPrepare(qcu_server server, int config_id);
/* Queues a solve of M(kappa, c_sw) x_r = b_r, r < nrhs (nrhs <= columns).
 * Returns at once; *ticket identifies the request. */
int qcuServerSubmit(qcu_server server, int config_id, double kappa, double csw, int nrhs, const void* b, void* x,
                    long long* ticket);
/* One pass of the request loop; never waits for the GPU. *finished receives
 * the number of requests that completed in this pass. */
int qcuServerPoll(qcu_server server, int* finished);
/* *finished = 1 once x holds the solution; then *latency_s is the time from
 * submission to completion, reports (nrhs entries) are filled and the request's
 * status is returned. */
int qcuServerQuery(qcu_server server, long long ticket, int* finished, double* latency_s, qcu_solve_report* reports);
/* Forgets a finished request. */
int qcuServerRelease(qcu_server server, long long ticket);
/* Runs a whole trace: request i is submitted arrival_s[i] seconds (non-
 * decreasing) after the call starts, and the loop polls until all finished.
 * latency_s[i] is measured from the scheduled arrival; reports (sum of nrhs
 * entries, in request order) may be NULL. */
int qcuServerRunTrace(qcu_server server, int n, const double* arrival_s, const int* config_id, const double* kappa,
                      const double* csw, const int* nrhs, const void* const* b, void* const* x, double* latency_s,
                      qcu_solve_report* reports);
/* Requests submitted and not yet finished. */
int qcuServerPending(qcu_server server);
/* Device bytes held by resident configurations. */
long long qcuServerDeviceBytes(qcu_server server);
/* Page-locked host memory for sources and solutions (NULL on failure). */
void* qcuHostAlloc(long long bytes);
void qcuHostFree(void* p);

/* Times the fused stencil kernel on resident internal fields: `variant`
 * 0 = hop only, 1 = hop + A^-1, 2 = hop + A^-1 + xpay + second output + norm
 * (the CG's K2), 3 = the CG update stencil, 4 = variant 2 without the norm
 * and its reduction; precision as above;
 * nrhs right-hand sides. Runs `iters` launches and returns the mean device
 * time per launch in milliseconds, measured with CUDA events on the
 * context stream; *bytes receives the algorithmic bytes of one launch. */
int qcuBenchStencil(qcu_context ctx, int precision, int variant, int nrhs, int iters, double* ms_per_launch,
                    double* bytes);

/* Autotuner: times the fused stencil over every launch shape (RHS lanes x
 * site lanes) for this precision and number of right-hand sides on the
 * context's lattice, keeps the fastest for the solver, and reports it. With
 * QCU_TUNE_CACHE=<file> the choice is appended to that file and reused. */
int qcuAutotune(qcu_context ctx, int precision, int nrhs, int* rhs_lanes, int* site_lanes, double* ms);

/* Number of kernels this library enqueued since the context was created. */
long long qcuContextLaunchCount(qcu_context ctx);

/* The context behind the reference interface (NULL before initGridSize). */
qcu_context qcuLegacyContext(void);

/* The reference's storage shifts (include/qcu_shift_storage.cuh:14-16,
 * src/qcu_shift_storage.cu:166-195), also exported under its C++ names
 * shiftVectorStorage / shiftGaugeStorage. direction 0 (TO_COALESCE): AoS ->
 * the reference's SoA; 1 (TO_NON_COALESCE): back. Spinor: one parity block,
 * [V/2][24 doubles] <-> [24][V/2]. Gauge: [4][2][V/2][9 complex] <->
 * [4][2][12][V/2] (first two rows; going back rebuilds the third as
 * conj(row0 x row1), where the reference's shift back does nothing). Device
 * pointers, lattice extents with Lx even; synchronous. */
int qcuShiftVectorStorage(void* dst, const void* src, int direction, int Lx, int Ly, int Lz, int Lt);
int qcuShiftGaugeStorage(void* dst, const void* src, int direction, int Lx, int Ly, int Lz, int Lt);

/* ---- domain decomposition along t (several GPUs, one lattice) ----
 * Replaces the reference's MPI communicator (src/qcu_communicator.cu:
 * 1033-1268 halo exchange, 1603-1623 global sums), which splits the lattice
 * over a process grid; here the split is along t only, one slab per rank
 * (one process per GPU), the local time extent Lt / nranks even and the time
 * slice (Lx/2 * Ly * Lz sites) a multiple of 32. Each parity block of every
 * field of a slab context carries two ghost slices behind its sites; before a
 * hop the slab's first and last slices are sent to the neighbouring ranks'
 * ghost slices (into the receiver's own memory), and the solver's dot
 * products are summed over the ranks. Fields given to a slab context are the
 * rank's part of the global field: the slices t0 .. t0 + Lt/nranks - 1, t0 =
 * rank * Lt/nranks, in the reference AoS layouts of that local lattice.
 *
 * Transports: NCCL (ncclSend/ncclRecv into the peers' ghost slices, and
 * ncclAllReduce, all enqueued on the context's stream, so CUDA graphs capture
 * them), or a host transport whose two callbacks move host buffers between
 * ranks (for callers that bring their own messaging, as the reference's MPI
 * host staging does; the library stages through pinned host memory and
 * synchronises around each call, and solves on it run without CUDA graphs). */
typedef struct qcu_comm_s* qcu_comm;
/* Host transport: send send_lo (this rank's first slices) to rank - 1 and
 * send_hi (its last slices) to rank + 1, receive rank + 1's send_lo into
 * recv_hi and rank - 1's send_hi into recv_lo (ranks modulo nranks; all four
 * buffers `bytes` long, host memory). Returns 0 on success. */
typedef int (*qcu_exchange_fn)(void* user, const void* send_lo, const void* send_hi, void* recv_lo, void* recv_hi,
                               size_t bytes);
/* Host transport: values[0..n) <- their sum over all ranks. Returns 0 on success. */
typedef int (*qcu_allreduce_fn)(void* user, double* values, int n);

/* The NCCL unique id (bytes >= 128) rank 0 creates and every rank passes to
 * qcuCommCreateNccl. */
int qcuCommNcclUniqueId(void* id, int bytes);
/* This process's rank of an NCCL communicator of nranks ranks on `device`. */
int qcuCommCreateNccl(qcu_comm* comm, const void* id, int nranks, int rank, int device);
int qcuCommCreateHost(qcu_comm* comm, int nranks, int rank, qcu_exchange_fn exchange, qcu_allreduce_fn allreduce,
                      void* user);
int qcuCommDestroy(qcu_comm comm);
/* The slab of the comm's rank of the global lattice `lattice` on `device`.
 * qcuLoadGauge / qcuGenerateGauge, qcuDslash, qcuApplyOperator and qcuInvert
 * work on it with local fields; every rank makes the same calls in the same
 * order. The context keeps an extended copy of its slab (two more slices on
 * each side) for the clover term. Not for the request server or the
 * reference-interface entry points. */
int qcuContextCreateSlab(qcu_context* ctx, const int lattice[4], qcu_comm comm, int device);
/* The slab geometry (host arithmetic only, no GPU): out = {t0, local Lt,
 * slice sites, local half volume, first forward-ghost site, first
 * backward-ghost site}; QCU_ERR_INVALID_ARG when the lattice does not split. */
int qcuSlabGeometry(const int lattice[4], int nranks, int rank, int out[6]);

/* Test hook for host-side fault injection: after n more successful device
 * allocations the next one fails as out-of-memory (n < 0 disables). */
void qcuDebugFailAllocAfter(long long n);

/* Test hook: batched launches of the fast 16-bit operator on the RHS-paired
 * kernels stage no neighbour words in shared memory (0), the t neighbours'
 * (1), the z and t neighbours' (2), or as built (-1), from the next launch on,
 * for the whole process. */
void qcuDebugSetPairStage(int stage);

/* Test hook: one launch of the batched stencil with epilogue flags `epi`
 * (1 A^-1 after the hop, 2 xpay, 4 A^-1 on x, 8 A^-1 after the xpay, 16 second
 * output A^-1 y, 32 per-RHS norm, 64 CG x/r update) on fields converted from
 * FP64 AoS spinors (nrhs x Vh x 12 complex, host or device memory; parity 0
 * output). csw_eff[r] <= 0 means no clover term for RHS r. out, out2, xacc
 * and racc are read before and written after the launch; norms[r] receives
 * the launch's per-RHS sums. rhs_pairs: 1 = RHS-paired kernels, 0 = one RHS
 * per thread, -1 = as built; the choice is process-wide for the duration of
 * the call, so this hook must not run concurrently with other solves. */
int qcuDebugStencil(qcu_context ctx, int precision, int dagger, int epi, int nrhs, const double* csw_eff,
                    const double* coef, const double* alpha, const int* active, const void* in, const void* x,
                    const void* pvec, void* out, void* out2, void* xacc, void* racc, double* norms,
                    int rhs_pairs);

#ifdef __cplusplus
}
#endif
#endif
