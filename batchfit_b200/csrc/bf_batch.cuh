// Device-side pieces shared by the mixed-batch kernels (bf_batch_kernels.cu,
// bf_batch_guess.cu).
#pragma once

#include "bf_batch.h"
#include "bf_lm.cuh"

namespace bf {

constexpr int kBatchBlock = 256;
constexpr int kBatchWarps = kBatchBlock / 32;
constexpr int kBatchMinBlocks = 2;
// Shared memory per warp: LM state (4 groups x 2 slots x K doubles, K <= 45) and
// the guess sorting buffer (two edge runs of kBatchMaxSortWidth floats per warp).
constexpr int kLmSlotDoubles = 2 * Layout<kTwoLorentzian>::K;
constexpr int kLmWarpDoubles = 4 * kLmSlotDoubles;
constexpr int kGuessWarpFloats = 2 * kBatchMaxSortWidth;
constexpr int kGuessSmem = kBatchWarps * kGuessWarpFloats * int(sizeof(float));
// The LM kernel runs 128-thread CTAs, 3 per SM: its two-Lorentzian classes need
// 168 registers (at 128 a thread they spill several KB of state).
constexpr int kBatchLmBlock = 128;
constexpr int kBatchLmMinBlocks = 3;
constexpr int kLmSmem = kBatchLmBlock / 32 * kLmWarpDoubles * int(sizeof(double));

// Claim the next item of a class for a group: lane 0 takes a ticket, all lanes
// get it.  False when the class is drained.
template <int G>
__device__ __forceinline__ bool claim(const Group<G> &g, unsigned long long *counter, const WorkClass &cls,
                                      const WorkItem *items, WorkItem &it) {
    unsigned long long t = 0;
    if (g.lane == 0)
        t = atomicAdd(counter, 1ull);
    t = g.bcast(t, 0);
    if (t >= (unsigned long long)cls.fits)
        return false;
    it = items[cls.begin + (long long)t];
    return true;
}

// The guess kernel (bf_batch_guess.cu): occupancy and launch.
cudaError_t batch_guess_blocks_per_sm(int *blocks);
void launch_batch_guess(const BatchArgs &b, int grid, cudaStream_t stream);

} // namespace bf
