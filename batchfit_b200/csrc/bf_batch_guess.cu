// Data-only guesses of a mixed batch: one persistent launch over every segment
// without p0 (bf_batch.h), each work class handled by its initial_guess
// instantiation (group lanes and register sort width chosen from M).
#include "bf_batch.cuh"

namespace bf {

namespace {

// ------------------------------------------------------------------ guess --
template <int MODEL, int G, int V>
__device__ __forceinline__ void guess_class(const BatchArgs &b, const WorkClass &cls, unsigned long long *counter,
                                            float *warp_buf) {
    constexpr int P = Model<MODEL>::P;
    const Group<G> g;
    float *scratch = warp_buf + ((threadIdx.x & 31u) / G) * (kGuessWarpFloats / (32 / G));
    WorkItem it;
    while (claim(g, counter, cls, b.guess_items, it)) {
        const Segment &seg = b.segs[it.segment];
        const int m = seg.a.m;
        const float *row = seg.a.y + (long long)it.fit * m;
        const bool vec_ok = (m & 3) == 0 && (reinterpret_cast<uintptr_t>(row) & 15) == 0;
        bool yfin, flat;
        float syy;
        stage_row<G, false>(g, row, m, vec_ok, nullptr, yfin, flat, syy);
        const XConst xc = seg.xc;
        float p[P];
        initial_guess<MODEL, G, V>(g, xc, seg.a.x, row, yfin, scratch, p);
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (int(g.lane) == k)
                seg.guesses[(long long)it.fit * P + k] = p[k];
        g.sync();
    }
}

__global__ void __launch_bounds__(kBatchBlock, kBatchMinBlocks) batch_guess_kernel(BatchArgs b) {
    extern __shared__ __align__(16) float guess_smem[];
    float *warp_buf = guess_smem + (threadIdx.x / 32) * kGuessWarpFloats;
    const int classes = b.hdr->guess_classes;
    unsigned long long *counters = b.counters + kMaxClasses;
    for (int c = 0; c < classes; ++c) {
        const WorkClass cls = b.guess_classes[c];
        switch (cls.model * 1000 + cls.lanes * 10 + (cls.v == 16 ? 2 : cls.v == 4 ? 1 : 0)) {
#define BF_GUESS_CASE(MODEL, G, V, CODE)                                                                       \
    case MODEL * 1000 + G * 10 + CODE: guess_class<MODEL, G, V>(b, cls, counters + c, warp_buf); break;
#define BF_GUESS_MODEL(MODEL)                                                                                  \
    BF_GUESS_CASE(MODEL, 8, 4, 1)                                                                              \
    BF_GUESS_CASE(MODEL, 8, 16, 2)                                                                             \
    BF_GUESS_CASE(MODEL, 16, 16, 2)                                                                            \
    BF_GUESS_CASE(MODEL, 32, 16, 2)                                                                            \
    BF_GUESS_CASE(MODEL, 32, 0, 0)
            BF_GUESS_MODEL(0)
            BF_GUESS_MODEL(1)
            BF_GUESS_MODEL(2)
            BF_GUESS_MODEL(3)
#undef BF_GUESS_MODEL
#undef BF_GUESS_CASE
        default: break;
        }
        __syncwarp();
    }
}

} // namespace

cudaError_t batch_guess_blocks_per_sm(int *blocks) {
    cudaError_t e = cudaFuncSetAttribute(batch_guess_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGuessSmem);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, batch_guess_kernel, kBatchBlock, kGuessSmem);
    return e;
}

void launch_batch_guess(const BatchArgs &b, int grid, cudaStream_t stream) {
    batch_guess_kernel<<<grid, kBatchBlock, kGuessSmem, stream>>>(b);
}

} // namespace bf
