// monitor.cuh -- the residual monitor and stop rules of projectGS on the
// device, for steps captured into one CUDA graph.
//
// simpleMonitorError (xpbdLayer3D.m:515-544) decides after every iteration
// whether the layer loop goes on; on the host that needs the residual back
// every iteration.  Here the loop of a layer is a conditional WHILE node of
// the step graph and each layer sits in a conditional IF node; single-thread
// kernels apply the same rules to a state kept in device memory and set the
// nodes' conditions (cudaGraphSetConditional).  The number of iterations of
// a layer is capped (MonState.error = 1 and the loop ends).
#pragma once

#include <cuda_runtime.h>

namespace mlx {

constexpr int kMonCapacity = 16384;         // residualArray entries per step
constexpr long long kMonMaxIterations = 1000000;  // per layer

struct MonParams {
  double stop_at_improvement_percent;
  double give_up_threshold;
  int give_up_enabled;
  int last_layer_give_up_enabled;
  long long hanging_stop;
};

struct MonState {
  double run_until;     // runUntilResSmallerThan (persists across steps)
  double set_percent;   // StopAtImprovementPercent still to apply (layer 1, first iteration)
  double normresv;      // ||residualv|| at the start of the layer (xpbdLayer3D.m:161)
  double res;           // residual of the last iteration
  int ra_len;
  int decreased;        // errorChangeDecreased
  int stop;             // stopSolve
  int end_layer;
  long long it;
  int total_iterations;
  int error;            // 1: iteration cap, 2: residualArray full
  double ra[kMonCapacity];
};

// integrate: residualArray = [initialResidual = 0] (xpbdLayer3D.m:670-674)
__global__ void k_mon_step_begin(MonState* ms) {
  ms->ra_len = 1;
  ms->ra[0] = 0.0;
  ms->decreased = 0;
  ms->stop = 0;
  ms->total_iterations = 0;
  ms->error = 0;
}

// Before a layer: the layer runs unless stopSolve is set (layerSolve's
// `break`, xpbdLayer3D.m:223-225); StopAtImprovementPercent applies to the
// first layer only.
__global__ void k_mon_layer_begin(MonState* ms, cudaGraphConditionalHandle run_layer, int layer, MonParams mp) {
  ms->set_percent = layer == 0 ? mp.stop_at_improvement_percent : 0.0;
  cudaGraphSetConditional(run_layer, ms->stop ? 0u : 1u);
}

// projectGS loop entry: it = 1, while it <= iterations || (~stopSolve &&
// runUntil >= 0 && lastLayer) (xpbdLayer3D.m:315).
__global__ void k_mon_loop_begin(MonState* ms, cudaGraphConditionalHandle loop, int iterations, int is_last) {
  ms->it = 1;
  ms->end_layer = 0;
  const bool go = 1 <= iterations || (!ms->stop && ms->run_until >= 0 && is_last);
  cudaGraphSetConditional(loop, go ? 1u : 0u);
}

// End of one projectGS iteration: append the residual and apply
// simpleMonitorError's rules (xpbdLayer3D.m:515-544), then the loop test.
// With ns_every > 0 it also sets `ns`, the condition of the Newton-PCG
// correction (pcg.cuh) that closes the iteration: after every ns_every
// iterations of the last layer, when the loop goes on.
__device__ __forceinline__ void mon_iter_end(MonState* ms, cudaGraphConditionalHandle loop, int iterations,
                                             int is_last, const MonParams& mp, cudaGraphConditionalHandle ns = 0,
                                             int ns_every = 0) {
  ms->it += 1;
  ms->total_iterations += 1;
  const double newRes = ms->res;
  if (ms->ra_len < kMonCapacity) {
    ms->ra[ms->ra_len++] = newRes;
  } else {
    ms->error = 2;
    ms->stop = 1;
  }
  const double lastResidual = fabs(ms->ra[ms->ra_len - 2]);
  const double newResidual = fabs(newRes);
  const double errorChange = newResidual - lastResidual;
  if (ms->set_percent > 0) {
    ms->run_until = fmax((1 - ms->set_percent / 100.0) * newResidual, 1e-8);
    ms->set_percent = 0;
  }
  if (errorChange < 0) ms->decreased = 1;
  if (mp.give_up_enabled && errorChange > mp.give_up_threshold && ms->decreased &&
      (!is_last || mp.last_layer_give_up_enabled))
    ms->end_layer = 1;
  const bool stopHanging = (long long)ms->ra_len > mp.hanging_stop && mp.hanging_stop >= 0;
  if (stopHanging ||
      (ms->run_until >= 0 && (ms->run_until >= newResidual && (is_last || ms->normresv < ms->run_until))))
    ms->stop = 1;
  if (ms->it > kMonMaxIterations) {
    ms->error = 1;
    ms->end_layer = 1;
  }
  const bool go = !(ms->end_layer || ms->stop) &&
                  (ms->it <= iterations || (!ms->stop && ms->run_until >= 0 && is_last));
  cudaGraphSetConditional(loop, go ? 1u : 0u);
  if (ns_every > 0) cudaGraphSetConditional(ns, (go && (ms->it - 1) % ns_every == 0) ? 1u : 0u);
}

__global__ void k_mon_iter_end(MonState* ms, cudaGraphConditionalHandle loop, int iterations, int is_last,
                               MonParams mp, cudaGraphConditionalHandle ns, int ns_every) {
  mon_iter_end(ms, loop, iterations, is_last, mp, ns, ns_every);
}

}  // namespace mlx
