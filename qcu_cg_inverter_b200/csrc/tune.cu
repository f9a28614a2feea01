// Launch-shape autotuner.
//
// For a (precision, number of right-hand sides) pair the tuner times the
// solver's heaviest kernel - the fused stencil hop + A^-1 + xpay + second
// output + norm - over every block shape (RHS lanes Rb in powers of two up to
// min(nrhs, 32), times 64/128/256 threads) on resident fields of the
// context's lattice, and keeps the fastest. The solver launches every kernel
// of that batch with the chosen shape. Results live in the context and, when
// QCU_TUNE_CACHE names a file, are appended there and reloaded by later
// contexts of the same lattice ("Lx Ly Lz Lt prec nrhs Rb Sb ms" per line).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "qcu_context.h"

namespace qcu {

static LaunchShape default_shape(int nrhs) {
  if (nrhs <= 1) return LaunchShape{1, 128};
  int rb = 1;
  while (rb * 2 <= nrhs && rb * 2 <= 8) rb *= 2;
  return LaunchShape{rb, 128 / rb};
}

static void load_cache(qcu_context ctx) {
  if (ctx->tune_cache_loaded) return;
  ctx->tune_cache_loaded = true;
  const char* path = getenv("QCU_TUNE_CACHE");
  if (!path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  int L[4], prec, nrhs, rb, sb;
  double ms;
  while (fscanf(f, "%d %d %d %d %d %d %d %d %lf", &L[0], &L[1], &L[2], &L[3], &prec, &nrhs, &rb, &sb, &ms) == 9) {
    if (memcmp(L, ctx->L, sizeof(L)) == 0) ctx->tuned[std::make_pair(prec, nrhs)] = LaunchShape{rb, sb};
  }
  fclose(f);
}

LaunchShape ctx_shape(qcu_context ctx, int prec, int nrhs) {
  load_cache(ctx);
  auto it = ctx->tuned.find(std::make_pair(prec, nrhs));
  if (it != ctx->tuned.end()) return it->second;
  return default_shape(nrhs);
}

bool ctx_is_tuned(qcu_context ctx, int prec, int nrhs) {
  load_cache(ctx);
  return ctx->tuned.count(std::make_pair(prec, nrhs)) != 0;
}

// `spinor_prec` is the public precision; the timed operator is the variant
// that serves it (ctx_op), and the result is kept under that variant.
int ctx_autotune(qcu_context ctx, int spinor_prec, int nrhs, double* best_ms) {
  const Geom& g = ctx->g;
  cudaStream_t st = ctx->stream;
  const int op = ctx_op(ctx, spinor_prec, nrhs);
  const int prec = op_spinor_prec(op);
  if (!ctx->gauge_loaded) {
    set_error(QCU_ERR_NOT_INITIALIZED, "no gauge field loaded");
    return QCU_ERR_NOT_INITIALIZED;
  }
  Field fin, fout, fx, fout2;
  QCU_CHECK(fin.alloc(prec, g.Vh_pad, nrhs, 1, st));
  QCU_CHECK(fout.alloc(prec, g.Vh_pad, nrhs, 1, st));
  QCU_CHECK(fx.alloc(prec, g.Vh_pad, nrhs, 1, st));
  QCU_CHECK(fout2.alloc(prec, g.Vh_pad, nrhs, 1, st));
  {
    DevBuf aos;
    QCU_CHECK(aos.ensure((size_t)g.Vh * 192 * nrhs, st));
    QCU_CHECK_CUDA(launch_spinor_random((size_t)g.Vh * nrhs, 5, aos.p, st));
    QCU_CHECK_CUDA(launch_spinor_in(prec, g, nrhs, aos.p, (size_t)g.Vh * 12, fin.view(0), st));
    QCU_CHECK_CUDA(launch_spinor_in(prec, g, nrhs, aos.p, (size_t)g.Vh * 12, fx.view(0), st));
    QCU_CHECK_CUDA(cudaStreamSynchronize(st));
  }
  int slot;
  QCU_CHECK(ctx_clover_slot(ctx, 0.13, &slot));
  QCU_CHECK(ctx->red.ensure(g, nrhs, st, 2));  // smallest candidate: 32 RHS lanes x 2 sites
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
  const int epi = EPI_CPRE | EPI_XPAY | EPI_OUT2 | EPI_NORM;
  cudaEvent_t e0, e1;
  QCU_CHECK_CUDA(cudaEventCreate(&e0));
  QCU_CHECK_CUDA(cudaEventCreate(&e1));
  LaunchShape best = default_shape(nrhs);
  double best_t = 1e30;
  for (int rb = 1; rb <= 32 && rb <= (nrhs >= 2 ? nrhs : 1); rb *= 2) {
    for (int threads : {64, 128, 256}) {
      if (threads % rb) continue;
      LaunchShape sh{rb, threads / rb};
      if (launch_dslash(op, false, epi, FIN_NONE, a, sh, st) != cudaSuccess) {
        (void)cudaGetLastError();
        continue;
      }
      QCU_CHECK_CUDA(launch_dslash(op, false, epi, FIN_NONE, a, sh, st));
      QCU_CHECK_CUDA(cudaEventRecord(e0, st));
      const int reps = 5;
      for (int k = 0; k < reps; k++) QCU_CHECK_CUDA(launch_dslash(op, false, epi, FIN_NONE, a, sh, st));
      QCU_CHECK_CUDA(cudaEventRecord(e1, st));
      QCU_CHECK_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      QCU_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      ctx->launches += reps + 2;
      if (ms / reps < best_t) {
        best_t = ms / reps;
        best = sh;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->tuned[std::make_pair(op, nrhs)] = best;
  if (best_ms) *best_ms = best_t;
  const char* path = getenv("QCU_TUNE_CACHE");
  if (path) {
    FILE* f = fopen(path, "a");
    if (f) {
      fprintf(f, "%d %d %d %d %d %d %d %d %.6f\n", ctx->L[0], ctx->L[1], ctx->L[2], ctx->L[3], op, nrhs, best.Rb,
              best.Sb, best_t);
      fclose(f);
    }
  }
  return QCU_SUCCESS;
}

}  // namespace qcu

using namespace qcu;

extern "C" int qcuAutotune(qcu_context ctx, int precision, int nrhs, int* rhs_lanes, int* site_lanes, double* ms) {
  clear_error();
  QCU_CHECK(ctx_check(ctx));
  if (precision < 0 || precision > 2 || nrhs < 1) {
    set_error(QCU_ERR_INVALID_ARG, "bad autotune arguments");
    return QCU_ERR_INVALID_ARG;
  }
  QCU_CHECK(ctx_autotune(ctx, precision, nrhs, ms));
  LaunchShape sh = ctx_shape(ctx, ctx_op(ctx, precision, nrhs), nrhs);
  if (rhs_lanes) *rhs_lanes = sh.Rb;
  if (site_lanes) *site_lanes = sh.Sb;
  return QCU_SUCCESS;
}
