// qcuBenchStencil (device timing of the fused stencil on resident fields) and
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
  if (prec < 0 || prec > 2 || variant < 0 || variant > 2 || nrhs < 1 || iters < 1) {
    set_error(QCU_ERR_INVALID_ARG, "bad benchmark arguments");
    return QCU_ERR_INVALID_ARG;
  }
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  const int op = ctx_op(ctx, prec);  // the operator variant the solver uses for this precision
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
  int slot = 0;
  if (variant >= 1) QCU_CHECK(ctx_clover_slot(ctx, 0.13, &slot));
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
  int epi = variant == 0 ? 0 : (variant == 1 ? EPI_CPRE : (EPI_CPRE | EPI_XPAY | EPI_OUT2 | EPI_NORM));
  for (int k = 0; k < 3; k++) QCU_CHECK_CUDA(launch_dslash(op, false, epi, FIN_NONE, a, sh, st));
  cudaEvent_t e0, e1;
  QCU_CHECK_CUDA(cudaEventCreate(&e0));
  QCU_CHECK_CUDA(cudaEventCreate(&e1));
  QCU_CHECK_CUDA(cudaEventRecord(e0, st));
  for (int k = 0; k < iters; k++) QCU_CHECK_CUDA(launch_dslash(op, false, epi, FIN_NONE, a, sh, st));
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
    if (variant == 2) per_rhs += 2.0 * spinor_b(prec);  // xpay input + second output
    double shared = 8.0 * link_b(op_link_format(op)) + (variant >= 1 ? clov_b(op_clover_prec(op)) : 0.0);
    int tiles = (nrhs + sh.Rb - 1) / sh.Rb;
    *bytes = (double)g.Vh * (nrhs * per_rhs + tiles * shared);
  }
  return QCU_SUCCESS;
}
