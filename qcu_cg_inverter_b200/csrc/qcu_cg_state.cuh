// Device-resident CG scalars, one entry per right-hand side, and the finishing
// functors that update them at the end of a fused reduction (executed by every
// thread of the last block, thread t of nt for RHS t, t + nt, ..., so no host
// round trip is needed per iteration and no thread walks all the RHS).
//
// Iteration of the sloppy CG on N = Mhat^dag Mhat (per RHS r):
//   y = Mhat p, pAp = |y|^2           -> FinCgAlpha: alpha = rr / pAp
//   z = Mhat^dag y
//   x += alpha p, r -= alpha z, rr' = |r|^2
//                                     -> FinCgBeta:  beta = rr'/rr, rr = rr';
//                                        pauses the RHS (active = 0, event = 1)
//                                        when rr' < trigger (reliable update or
//                                        convergence check due)
//   p = r + beta p
// The reference computes alpha and beta on the host after two blocking copies
// per dot product (src/cg_inverter.cu:204-235); here they never leave the GPU.
#pragma once
#include "qcu_common.cuh"

namespace qcu {

struct CgDevState {
  double* rr;       // |r|^2 of the iterated residual
  double* rr_old;   // |r|^2 before the last update (for beta after a reliable update)
  double* pAp;
  double* alpha;
  double* beta;
  double* trigger;  // pause when rr < trigger
  int* active;      // 1 while the RHS iterates
  int* event;       // set when the RHS paused itself
  int* iters;
  int* breakdown;   // set when pAp <= 0 or not finite
  int* final_trig;  // 1 when the trigger is the convergence target
  // when one RHS pauses for its reliable update, every other iterating RHS
  // whose |r|^2 is within this factor of its own (non-final) trigger pauses
  // with it, so that their updates coincide (1: off)
  double align;
  // the reliable update's stopping rule (rel_stop) and its inputs
  const double* bnorm;  // |b|
  const int* upd;       // RHS in the current reliable update
  int* cont;            // out: RHS of the update that go on
  double tol;
  int maxiter;
};

// Why a reliable update ends a RHS's solve, from its true residual |A r|^2
// (|r|^2 without clover): REL_GO, it goes on. The residual |A r| / |b| is
// left in *res.
enum { REL_GO = 0, REL_CONV, REL_BREAK, REL_CAP };
QCU_D int rel_stop(double ar2, double bn, int brk, int iters, double tol, int maxiter, double* res) {
  *res = bn > 0 ? sqrt(fmax(ar2, 0.0)) / bn : 0.0;
  if (bn == 0.0 || *res < tol) return REL_CONV;
  if (!isfinite(*res) || brk) return REL_BREAK;
  if (iters >= maxiter) return REL_CAP;
  return REL_GO;
}

// Finishing functor of the true-residual reduction of a reliable update:
// marks the RHS that go on, so that only they get r_ne.
struct FinRelCont {
  static QCU_D void apply(const double* res, int nrhs, int NR, void* st, int t, int nt) {
    CgDevState* s = static_cast<CgDevState*>(st);
    for (int r = t; r < nrhs; r += nt) {
      double q;
      s->cont[r] = s->upd[r] && rel_stop(res[r * NR], s->bnorm[r], s->breakdown[r], s->iters[r], s->tol,
                                         s->maxiter, &q) == REL_GO;
    }
  }
};

// Every thread of the block calls apply (t = its index, nt = the block's
// threads): FinCgBeta has a block barrier.
struct FinCgAlpha {
  static QCU_D void apply(const double* res, int nrhs, int NR, void* st, int t, int nt) {
    CgDevState* s = static_cast<CgDevState*>(st);
    for (int r = t; r < nrhs; r += nt) {
      if (!s->active[r]) continue;
      double pap = res[r * NR];
      s->pAp[r] = pap;
      if (!(pap > 0.0) || !isfinite(pap)) {
        s->breakdown[r] = 1;
        s->active[r] = 0;
        s->event[r] = 1;
        s->alpha[r] = 0.0;
      } else {
        s->alpha[r] = s->rr[r] / pap;
      }
    }
  }
};

struct FinCgBeta {
  static QCU_D void apply(const double* res, int nrhs, int NR, void* st, int t, int nt) {
    CgDevState* s = static_cast<CgDevState*>(st);
    bool paused = false;
    for (int r = t; r < nrhs; r += nt) {
      if (!s->active[r]) continue;
      double rn = res[r * NR];
      s->beta[r] = rn / s->rr[r];
      s->rr_old[r] = s->rr[r];
      s->rr[r] = rn;
      s->iters[r] += 1;
      if (!isfinite(rn)) {
        s->breakdown[r] = 1;
        s->active[r] = 0;
        s->event[r] = 1;
      } else if (rn < s->trigger[r]) {
        s->active[r] = 0;
        s->event[r] = 1;
        paused = true;
      }
    }
    // a thread reads back only its own RHS below: the barrier only has to
    // tell every thread whether any RHS paused
    if (__syncthreads_or(paused) && s->align > 1.0) {
      for (int r = t; r < nrhs; r += nt) {
        if (s->active[r] && !s->final_trig[r] && s->rr[r] < s->align * s->trigger[r]) {
          s->active[r] = 0;
          s->event[r] = 1;
        }
      }
    }
  }
};

}  // namespace qcu
