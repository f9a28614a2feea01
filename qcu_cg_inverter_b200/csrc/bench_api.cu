// qcuBenchStencil (device timing of the fused stencil on resident fields),
// qcuDebugStencil (one stencil launch on converted fields, for tests) and
// qcuExportGauge.
#include <string.h>

#include "qcu_context.h"

namespace qcu {

__global__ void gauge_internal_to_aos_kernel(Geom g, const void* src64, double2* aos) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 8 * g.Vh) return;
  const int mp = l / g.Vh, s = l - mp * g.Vh;
  Link<double> U;
  LinkIO<PREC_DOUBLE>::load(U, src64, g.Vh_pad, mp >> 1, mp & 1, s);
  for (int k = 0; k < 9; k++) aos[(size_t)l * 9 + k] = make_double2(U.u[k].re, U.u[k].im);
}

}  // namespace qcu

using namespace qcu;

extern "C" int qcuExportGauge(qcu_context ctx, void* out) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (!out || !ctx->gauge_loaded) {
    set_error(QCU_ERR_INVALID_ARG, "no gauge field or null output");
    return QCU_ERR_INVALID_ARG;
  }
  size_t bytes = (size_t)8 * ctx->g.Vh * 9 * 16;
  bool dev = is_device_ptr(out);
  void* dst = out;
  if (!dev) {
    QCU_CHECK(ctx->stage_out.ensure(bytes, ctx->stream));
    dst = ctx->stage_out.p;
  }
  gauge_internal_to_aos_kernel<<<(8 * ctx->g.Vh + 127) / 128, 128, 0, ctx->stream>>>(ctx->g, ctx->gauge64.p,
                                                                                      static_cast<double2*>(dst));
  QCU_CHECK_CUDA(cudaGetLastError());
  ctx->launches++;
  if (!dev) QCU_CHECK_CUDA(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  QCU_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
  return QCU_SUCCESS;
}

static int spinor_b(int prec) { return prec == PREC_DOUBLE ? 192 : (prec == PREC_SINGLE ? 96 : 52); }
static int link_b(int fmt) {
  return fmt == PREC_DOUBLE ? 96 : (fmt == PREC_SINGLE ? 48 : (fmt == PREC_HALF ? 24 : 72));  // 18 FP32 reals
}
static int clov_b(int prec) { return prec == PREC_DOUBLE ? 576 : (prec == PREC_SINGLE ? 288 : 148); }

extern "C" int qcuBenchStencil(qcu_context ctx, int prec, int variant, int nrhs, int iters, double* ms_per_launch,
                               double* bytes) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (prec < 0 || prec > 2 || variant < 0 || variant > 4 || nrhs < 1 || iters < 1) {
    set_error(QCU_ERR_INVALID_ARG, "bad benchmark arguments");
    return QCU_ERR_INVALID_ARG;
  }
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  const int op = ctx_op(ctx, prec, nrhs);  // the operator variant the solver uses for this precision
  Field fin, fout, fx, fout2;
  QCU_CHECK(fin.alloc(prec, g.Vh_pad, nrhs, 1, st));
  QCU_CHECK(fout.alloc(prec, g.Vh_pad, nrhs, 1, st));
  QCU_CHECK(fx.alloc(prec, g.Vh_pad, nrhs, 1, st));
  QCU_CHECK(fout2.alloc(prec, g.Vh_pad, nrhs, 1, st));
  {
    DevBuf aos;
    QCU_CHECK(aos.ensure((size_t)g.Vh * 192 * nrhs, st));
    QCU_CHECK_CUDA(launch_spinor_random((size_t)g.Vh * nrhs, 77, aos.p, st));
    QCU_CHECK_CUDA(launch_spinor_in(prec, g, nrhs, aos.p, (size_t)g.Vh * 12, fin.view(0), st));
    QCU_CHECK_CUDA(launch_spinor_random((size_t)g.Vh * nrhs, 78, aos.p, st));
    QCU_CHECK_CUDA(launch_spinor_in(prec, g, nrhs, aos.p, (size_t)g.Vh * 12, fx.view(0), st));
    QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  }
  // variant 3 (the CG update stencil): FP32 (FP64) x and r, a search direction
  // and per-RHS alpha
  const int pa = acc_prec(prec);
  Field fxa, fra, fp;
  DevBuf alpha;
  if (variant == 3) {
    QCU_CHECK(fxa.alloc(pa, g.Vh_pad, nrhs, 1, st));
    QCU_CHECK(fra.alloc(pa, g.Vh_pad, nrhs, 1, st));
    QCU_CHECK(fp.alloc(prec, g.Vh_pad, nrhs, 1, st));
    DevBuf aos;
    QCU_CHECK(aos.ensure((size_t)g.Vh * 192 * nrhs, st));
    QCU_CHECK_CUDA(launch_spinor_random((size_t)g.Vh * nrhs, 79, aos.p, st));
    QCU_CHECK_CUDA(launch_spinor_in(pa, g, nrhs, aos.p, (size_t)g.Vh * 12, fxa.view(0), st));
    QCU_CHECK_CUDA(launch_spinor_in(pa, g, nrhs, aos.p, (size_t)g.Vh * 12, fra.view(0), st));
    QCU_CHECK_CUDA(launch_spinor_in(prec, g, nrhs, aos.p, (size_t)g.Vh * 12, fp.view(0), st));
    std::vector<double> al(nrhs, 1e-3);  // small steps: the fields stay bounded over many launches
    QCU_CHECK(alpha.ensure(sizeof(double) * nrhs, st));
    QCU_CHECK_CUDA(cudaMemcpyAsync(alpha.p, al.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, st));
    QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  }
  int slot = 0;
  if (variant == 1 || variant == 2 || variant == 4) QCU_CHECK(ctx_clover_slot(ctx, 0.13, &slot));
  // the shape the solver would use (tuned when qcuAutotune ran, else the
  // default), unless qcuContextSetShape overrode the single-RHS shape
  LaunchShape sh = (nrhs == 1 && ctx->shape_set) ? ctx->shape1 : ctx_shape(ctx, op, nrhs);
  QCU_CHECK(ctx->red.ensure(g, nrhs, st, sh.Sb));
  DslashArgs a;
  memset(&a, 0, sizeof(a));
  a.g = g;
  a.parity = 0;
  a.nrhs = nrhs;
  a.in = fin.cview(0);
  a.out = fout.view(0);
  a.x = fx.cview(0);
  a.out2 = fout2.view(0);
  a.gauge = ctx_gauge(ctx, op);
  a.clover = static_cast<const char*>(ctx_clover_ptr(ctx, op, true)) + ctx_clover_stride(ctx, op) * slot;
  a.coef0 = -0.0169;
  a.bc_t = -1.0;
  a.red = ctx->red.args();
  if (variant == 3) {
    a.xacc = fxa.view(0);
    a.racc = fra.view(0);
    a.pvec = fp.cview(0);
    a.alpha = alpha.as<double>();
  }
  const int epi = variant == 0   ? 0
                  : variant == 1 ? EPI_CPRE
                  : variant == 2 ? (EPI_CPRE | EPI_XPAY | EPI_OUT2 | EPI_NORM)
                  : variant == 4 ? (EPI_CPRE | EPI_XPAY | EPI_OUT2)
                                 : (EPI_XPAY | EPI_CGXR);
  const bool dag = variant == 3;  // the CG update stencil applies D^dag
  for (int k = 0; k < 3; k++) QCU_CHECK_CUDA(launch_dslash(op, dag, epi, FIN_NONE, a, sh, st));
  cudaEvent_t e0, e1;
  QCU_CHECK_CUDA(cudaEventCreate(&e0));
  QCU_CHECK_CUDA(cudaEventCreate(&e1));
  QCU_CHECK_CUDA(cudaEventRecord(e0, st));
  for (int k = 0; k < iters; k++) QCU_CHECK_CUDA(launch_dslash(op, dag, epi, FIN_NONE, a, sh, st));
  QCU_CHECK_CUDA(cudaEventRecord(e1, st));
  QCU_CHECK_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  QCU_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->launches += 3 + iters;
  if (ms_per_launch) *ms_per_launch = (double)ms / iters;
  if (bytes) {
    double per_rhs = 8.0 * spinor_b(prec) + spinor_b(prec);
    if (variant == 2 || variant == 4) per_rhs += 2.0 * spinor_b(prec);  // xpay input + second output
    if (variant == 3) per_rhs += 2.0 * spinor_b(prec) - spinor_b(prec) + 4.0 * spinor_b(pa);  // x, p in; no out; x, r in and out
    double shared = 8.0 * link_b(op_link_format(op)) +
                    ((variant == 1 || variant == 2 || variant == 4) ? clov_b(op_clover_prec(op)) : 0.0);
    int tiles = (nrhs + sh.Rb - 1) / sh.Rb;
    *bytes = (double)g.Vh * (nrhs * per_rhs + tiles * shared);
  }
  return QCU_SUCCESS;
}

// One launch of a batched stencil on internal fields converted from AoS
// spinors (FP64, nrhs x Vh x 12 complex each): the comparison point of the
// kernel families against each other and against the CPU operator.
extern "C" int qcuDebugStencil(qcu_context ctx, int prec, int dagger, int epi, int nrhs, const double* csw_eff,
                               const double* coef, const double* alpha, const int* active, const void* in,
                               const void* x, const void* pvec, void* out, void* out2, void* xacc, void* racc,
                               double* norms, int rhs_pairs) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  const int known = EPI_CPRE | EPI_XPAY | EPI_CX | EPI_CPOST | EPI_OUT2 | EPI_NORM | EPI_CGXR;
  const bool cgxr = (epi & EPI_CGXR) != 0;
  if (prec < 0 || prec > 2 || nrhs < 1 || (epi & ~known) || !csw_eff || !coef || !in ||
      ((epi & EPI_XPAY) && !x) || (!cgxr && !out) || ((epi & EPI_OUT2) && !out2) ||
      (cgxr && (!xacc || !racc || !pvec || !alpha)) || rhs_pairs < -1 || rhs_pairs > 1) {
    set_error(QCU_ERR_INVALID_ARG, "bad stencil arguments");
    return QCU_ERR_INVALID_ARG;
  }
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  if (ctx->g.tdd) {
    set_error(QCU_ERR_UNSUPPORTED, "qcuDebugStencil runs on whole-lattice contexts only");
    return QCU_ERR_UNSUPPORTED;
  }
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  const int op = ctx_op(ctx, prec, nrhs);
  const int ps = op_spinor_prec(op);
  const int pa = acc_prec(ps);
  const size_t per = (size_t)g.Vh * 12;  // complex numbers per AoS spinor
  const size_t aos_bytes = per * 16 * nrhs;
  Field fin, fx, fp, fout, fout2, fxa, fra;
  DevBuf aos, dcoef, dalpha, dact, dcidx;
  QCU_CHECK(aos.ensure(aos_bytes, st));
  auto ingest = [&](Field& f, int fp_prec, const void* src) -> int {
    QCU_CHECK(f.alloc(fp_prec, g.Vh_pad, nrhs, 1, st));
    QCU_CHECK_CUDA(cudaMemcpyAsync(aos.p, src, aos_bytes, cudaMemcpyDefault, st));
    QCU_CHECK_CUDA(launch_spinor_in(fp_prec, g, nrhs, aos.p, per, f.view(0), st));
    return QCU_SUCCESS;
  };
  auto egress = [&](const Field& f, void* dst) -> int {
    QCU_CHECK_CUDA(launch_spinor_out(f.prec, g, nrhs, f.cview(0), aos.p, per, st));
    QCU_CHECK_CUDA(cudaMemcpyAsync(dst, aos.p, aos_bytes, cudaMemcpyDefault, st));
    return QCU_SUCCESS;
  };
  QCU_CHECK(ingest(fin, ps, in));
  if (epi & EPI_XPAY) QCU_CHECK(ingest(fx, ps, x));
  if (cgxr) {
    QCU_CHECK(ingest(fp, ps, pvec));
    QCU_CHECK(ingest(fxa, pa, xacc));
    QCU_CHECK(ingest(fra, pa, racc));
  } else {
    QCU_CHECK(ingest(fout, ps, out));
  }
  if (epi & EPI_OUT2) QCU_CHECK(ingest(fout2, ps, out2));
  // per-RHS clover fields (csw_eff <= 0: none), pinned while later values are
  // built so that none evicts another; coefficients and mask
  std::vector<int> cidx(nrhs, -1), act(nrhs, 1);
  auto unpin = [&]() {
    for (int r = 0; r < nrhs; r++)
      if (cidx[r] >= 0 && ctx->clover.pinned[cidx[r]] > 0) ctx->clover.pinned[cidx[r]] -= 1;
  };
  for (int r = 0; r < nrhs; r++) {
    if (csw_eff[r] > 0.0) {
      const int st_slot = ctx_clover_slot(ctx, csw_eff[r], &cidx[r]);
      if (st_slot != QCU_SUCCESS) {
        cidx[r] = -1;
        unpin();
        return st_slot;
      }
      ctx->clover.pinned[cidx[r]] += 1;
    }
    if (active) act[r] = active[r] != 0;
  }
  unpin();  // every value is built; the launch below reads them in order
  QCU_CHECK(dcoef.ensure(sizeof(double) * nrhs, st));
  QCU_CHECK(dalpha.ensure(sizeof(double) * nrhs, st));
  QCU_CHECK(dact.ensure(sizeof(int) * nrhs, st));
  QCU_CHECK(dcidx.ensure(sizeof(int) * nrhs, st));
  QCU_CHECK_CUDA(cudaMemcpyAsync(dcoef.p, coef, sizeof(double) * nrhs, cudaMemcpyHostToDevice, st));
  if (alpha) QCU_CHECK_CUDA(cudaMemcpyAsync(dalpha.p, alpha, sizeof(double) * nrhs, cudaMemcpyHostToDevice, st));
  QCU_CHECK_CUDA(cudaMemcpyAsync(dact.p, act.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
  QCU_CHECK_CUDA(cudaMemcpyAsync(dcidx.p, cidx.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, st));
  const LaunchShape sh = ctx_shape(ctx, op, nrhs);
  QCU_CHECK(ctx->red.ensure(g, nrhs, st, sh.Sb));
  DslashArgs a;
  memset(&a, 0, sizeof(a));
  a.g = g;
  a.parity = 0;
  a.nrhs = nrhs;
  a.in = fin.cview(0);
  if (!cgxr) a.out = fout.view(0);
  if (epi & EPI_XPAY) a.x = fx.cview(0);
  if (epi & EPI_OUT2) a.out2 = fout2.view(0);
  a.gauge = ctx_gauge(ctx, op);
  a.clover = ctx_clover_ptr(ctx, op, true);
  a.clover_stride = ctx_clover_stride(ctx, op);
  a.clover_idx = dcidx.as<int>();
  a.coef = dcoef.as<double>();
  a.bc_t = -1.0;
  a.active = dact.as<int>();
  a.red = ctx->red.args();
  if (cgxr) {
    a.xacc = fxa.view(0);
    a.racc = fra.view(0);
    a.pvec = fp.cview(0);
    a.alpha = dalpha.as<double>();
  }
  set_rhs_pairs_override(rhs_pairs);
  const cudaError_t e = launch_dslash(op, dagger != 0, epi, FIN_NONE, a, sh, st);
  set_rhs_pairs_override(-1);
  if (e == cudaErrorInvalidValue) {
    set_error(QCU_ERR_INVALID_ARG, "no stencil kernel for this epilogue");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK_CUDA(e);
  ctx->launches++;
  if (cgxr) {
    QCU_CHECK(egress(fxa, xacc));
    QCU_CHECK(egress(fra, racc));
  } else {
    QCU_CHECK(egress(fout, out));
  }
  if (epi & EPI_OUT2) QCU_CHECK(egress(fout2, out2));
  if (norms && (epi & (EPI_NORM | EPI_CGXR)))
    QCU_CHECK_CUDA(cudaMemcpyAsync(norms, ctx->red.result.p, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
  QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  return QCU_SUCCESS;
}
