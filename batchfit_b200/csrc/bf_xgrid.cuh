// Constants of a shared x grid computed by one warp straight from global memory,
// for kernels that do not stage x in shared memory (mixed batches, long spectra).
#pragma once

#include "bf_args.h"
#include "bf_device.cuh"

namespace bf {

// Grid constants of an x grid, computed by one warp: the same values
// cta_prologue derives for a CTA-staged grid (solver.hpp:58-69,223-239;
// initial_guess.hpp:131-153).
__device__ __forceinline__ XConst xconst_warp(const float *x, int m) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned min_abs = 0x7f800000u, min_diff = 0x7f800000u;
    bool fin = true, up = true, down = true, strict = true, varied = false;
    const float x0 = __ldg(x);
    // Unrolled so that the loads of several iterations are in flight together (the
    // loop is latency-bound on them otherwise: one warp per segment, M/32 rounds).
#pragma unroll 8
    for (int j = int(lane); j < m; j += 32) {
        const float v = __ldg(x + j);
        fin = fin && isfinite(v);
        varied = varied || v != x0;
        if (j > 0) {
            const float prev = __ldg(x + j - 1);
            const float d = v - prev;
            up = up && d >= 0.0f;
            down = down && d <= 0.0f;
            if (d != 0.0f && isfinite(d))
                min_abs = min(min_abs, __float_as_uint(fabsf(d)));
            strict = strict && v > prev;
            if (d > 0.0f)
                min_diff = min(min_diff, __float_as_uint(d));
        }
    }
    XConst xc;
    fin = __all_sync(0xffffffffu, fin);
    up = __all_sync(0xffffffffu, up);
    down = __all_sync(0xffffffffu, down);
    strict = __all_sync(0xffffffffu, strict);
    varied = __any_sync(0xffffffffu, varied);
    min_abs = __reduce_min_sync(0xffffffffu, min_abs);
    min_diff = __reduce_min_sync(0xffffffffu, min_diff);
    xc.m = m;
    xc.x_finite = fin;
    xc.varied_x = varied;
    const float spacing = __uint_as_float(min_abs);
    xc.spacing = (up || down) && isfinite(spacing) ? spacing : 0.0f;
    const int count = edge_count(m);
    xc.count = count;
    xc.n1 = pow2_at_least(count);
    xc.guess_ok = m >= 5 && fin && strict && isfinite(rsub(__ldg(x + m - 1), x0));
    xc.guess_spacing = __uint_as_float(min_diff);
    xc.left_x = midpoint_rn(__ldg(x + (count - 1) / 2), __ldg(x + count / 2));
    xc.right_x = midpoint_rn(__ldg(x + m - count + (count - 1) / 2), __ldg(x + m - count + count / 2));
    return xc;
}

} // namespace bf
