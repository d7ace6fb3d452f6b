// Convergence test of the FDM refinement loop (shared by the standalone
// test kernel in fdm.cu and the residual kernel's fused tail in cg.cu):
// iteration count, the residual tests (RTOL, ATOL, DTOL, NANORINF, ITS) and
// stagnation (three steps without a 10% gain on the best residual: the
// rounding floor, or a low precision too coarse for the operator), then the
// loop's while-condition. res0 is the squared residual norm.
#pragma once
#include "common.cuh"

namespace seg {

// The loop's set-up from res0, the squared norm of the right-hand side:
// rnorm0, the tolerance, the iteration-0 test; sets the while-condition
// (1 = iterate).
__device__ __forceinline__ void fdm_init_state(const FdmParams* __restrict__ p,
                                               FdmState* __restrict__ st, double res0,
                                               cudaGraphConditionalHandle h) {
  const double dp = sqrt(fabs(res0));
  st->rnorm0 = dp;
  st->ttol = fmax(p->rtol * dp, p->atol);
  st->dp = dp;
  st->best = dp;
  st->its = 0;
  st->stalled = 0;
  st->kerr = 0;
  int reason = 0;
  if (!(dp == dp) || isinf(dp)) reason = -9;
  else if (dp <= st->ttol) reason = dp < p->atol ? 3 : 2;
  else if (p->max_it <= 0) reason = -3;
  st->reason = reason;
  cudaGraphSetConditional(h, reason == 0 ? 1u : 0u);
}

__device__ __forceinline__ void fdm_check_state(const FdmParams* __restrict__ p,
                                                FdmState* __restrict__ st, double res0,
                                                cudaGraphConditionalHandle h) {
  // a loop already decided (the initial test, before a first step that the
  // solve graph runs unconditionally): the decision and count stand
  if (st->reason != 0) {
    cudaGraphSetConditional(h, 0u);
    return;
  }
  const double dp = sqrt(fabs(res0));
  const int its = st->its + 1;
  st->its = its;
  st->dp = dp;
  int reason = 0;
  if (!(dp == dp) || isinf(dp)) {
    reason = -9;
  } else if (dp <= st->ttol) {
    reason = dp < p->atol ? 3 : 2;
  } else if (dp >= p->dtol * st->rnorm0) {
    reason = -4;
  } else {
    if (dp > 0.9 * st->best) {
      if (++st->stalled >= 3) reason = -5;
    } else {
      st->stalled = 0;
    }
    if (!reason && its >= p->max_it) reason = -3;
  }
  st->best = fmin(st->best, dp);
  st->reason = reason;
  cudaGraphSetConditional(h, reason == 0 ? 1u : 0u);
}

}  // namespace seg
