// tune.cuh -- autotuner of the grid sums (opening ratio, brick shape).
#pragma once

#include "common.cuh"

namespace dwg {

// points_dev: one normalised cloud; prm: its flags (in_normal 3).  Runs
// warm_iters DWG iterations, then picks the fastest (beta, tile) whose RMS
// error against exact sums at `samples` seeded grid samples is <= tol.
int autotune(const float* points_dev, int n, const dwg_params& prm, float tol, int samples, int warm_iters,
             cudaStream_t stream, dwg_tune_result* out);

}  // namespace dwg
