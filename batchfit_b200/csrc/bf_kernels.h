// Host-side entry points into the fit kernels (implemented in bf_kernels.cu).
#pragma once

#include "bf_args.h"

namespace bf {

// Launch the persistent fit kernel for `model` with `lanes` (8, 16 or 32) lanes per
// fit on `stream`.  The caller zeroes a.work_counter (when non-null) beforehand.
cudaError_t launch_fit(int model, int lanes, const FitArgs &a, const GuessArgs &ga, int sms,
                       cudaStream_t stream, LaunchInfo *info);

// Dynamic shared memory of one CTA for (model, lanes, M).
int smem_bytes(int model, int lanes, int m);

// Largest M the shared-memory layout supports for `model`.
int max_points(int model);

} // namespace bf
