// Persistent kernels of a mixed batch (bf_batch.h): spectra of uneven M and mixed
// models in one launch per kernel, fed from a device work queue.
//
// Spectra are not staged in shared memory: with uneven M no fixed per-group buffer
// fits every fit, so the kernels read x and y through the L1 cache (read-only
// loads).  A fit's working set (its y row and x grid) stays resident in L1/L2 for
// the passes of its LM iterations; y comes from HBM once per kernel.
//
// Every warp walks the class list in order.  For each class it runs the class's
// template instantiation: its groups claim work items through the class's atomic
// counter until the class is drained, then the warp moves on.  There is no
// block-wide synchronisation, so warps drift between classes freely.
#include "bf_batch.cuh"
#include "bf_xgrid.cuh"

#include <mutex>

namespace bf {

namespace {

// Per segment: the x-grid constants.  Per run: one work item per fit.
__global__ void __launch_bounds__(kBatchBlock) batch_prepare_kernel(BatchArgs b) {
    const BatchHeader h = *b.hdr;
    const int warp = int(blockIdx.x) * kBatchWarps + int(threadIdx.x / 32);
    const int warps = int(gridDim.x) * kBatchWarps;
    for (int s = warp; s < h.segments; s += warps) {
        const XConst xc = xconst_warp(b.segs[s].a.x, b.segs[s].a.m);
        if ((threadIdx.x & 31u) == 0u)
            b.segs[s].xc = xc;
    }
    const int runs = h.lm_runs + h.guess_runs;
    for (int r = int(blockIdx.x); r < runs; r += int(gridDim.x)) {
        const bool lm = r < h.lm_runs;
        const WorkRun run = lm ? b.lm_runs[r] : b.guess_runs[r - h.lm_runs];
        WorkItem *items = lm ? b.lm_items : b.guess_items;
        for (long long i = threadIdx.x; i < run.count; i += kBatchBlock)
            items[run.start + i] = WorkItem{run.segment, int(run.first + i)};
    }
}

// --------------------------------------------------------------------- LM --
// The round loop of lm_kernel over a class's items: one fused pass per round,
// then the FP64 control; a finished group claims its next item.
template <int MODEL, int G>
__device__ __forceinline__ void lm_class(const BatchArgs &b, const WorkClass &cls, unsigned long long *counter,
                                         double *state) {
    constexpr int P = Model<MODEL>::P;
    constexpr int K = Layout<MODEL>::K;
    const Group<G> g;
    LmState<MODEL> s;
    const Segment *seg = nullptr;
    const float *row = nullptr;
    int fit = -1;
    bool flat = false;
    float syy = 0.0f;
    while (true) {
        if (fit < 0) {
            // Intake: claim items until one needs a pass or the class is drained.
            WorkItem it;
            while (claim(g, counter, cls, b.lm_items, it)) {
                seg = &b.segs[it.segment];
                const FitArgs &a = seg->a;
                const int m = a.m;
                row = a.y + (long long)it.fit * m;
                const bool vec_ok = (m & 3) == 0 && (reinterpret_cast<uintptr_t>(row) & 15) == 0;
                bool yfin;
                stage_row<G, false>(g, row, m, vec_ok, nullptr, yfin, flat, syy);
                bool init_finite = true;
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    s.p[k] = a.p0[(long long)it.fit * P + k];
                    init_finite = init_finite && isfinite(s.p[k]);
                }
                if (a.options_ok && init_finite && seg->xc.x_finite && yfin) {
                    lm_begin<MODEL>(a, s);
                    fit = it.fit;
                    break;
                }
                // Preflight rejection (solver.hpp:205-226): parameters keep the initial values.
                s.status = kInvalid;
                s.iterations = 0;
                s.chi2 = __longlong_as_double(0x7ff8000000000000ll);
                write_fit<MODEL>(g, a, it.fit, s);
            }
            if (fit < 0)
                break;
        }
        const FitArgs &a = seg->a;
        const XConst xc = seg->xc;
        const bool pass_finite = lm_pass<MODEL, G, false>(g, a.x, row, a.m, s.t, state + (1 - s.cur) * K);
        bool done = lm_after_pass<MODEL>(g, a, xc, flat, pass_finite, state, s);
        if (!done)
            done = lm_plan<MODEL>(a, xc, double(syy), state, s);
        if (done) {
            write_fit<MODEL>(g, a, fit, s);
            if (a.uncertainties && s.status == kConverged)
                write_information<MODEL>(g, a, fit, state + s.cur * K);
            g.sync();
            fit = -1;
        }
    }
}

// One LM kernel per work-class type (model, lanes per fit), each walking only its
// own classes: a kernel holding several instantiations spills (1.5-2.2 KB of
// stack), one holding a single instantiation keeps lm_kernel's registers.
template <int MODEL, int G>
__global__ void __launch_bounds__(kBatchLmBlock, MODEL == kTwoLorentzian ? 3 : 4) batch_lm_kernel(BatchArgs b) {
    extern __shared__ __align__(16) double lm_smem[];
    double *warp_state = lm_smem + (threadIdx.x / 32) * kLmWarpDoubles;
    const int classes = b.hdr->lm_classes;
    const int group = int(threadIdx.x & 31u) / G;
    double *state = warp_state + group * kLmSlotDoubles;
    for (int c = 0; c < classes; ++c) {
        const WorkClass cls = b.lm_classes[c];
        if (cls.model == MODEL && cls.lanes == G)
            lm_class<MODEL, G>(b, cls, b.counters + c, state);
        __syncwarp();
    }
}

// ------------------------------------------------------------- covariance --
// One thread per LM work item; items of segments without uncertainties are skipped.
__global__ void __launch_bounds__(128) batch_covariance_kernel(BatchArgs b) {
    if (b.hdr->uncertain_segments == 0)
        return;
    const long long items = b.hdr->lm_items;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < items;
         t += (long long)gridDim.x * blockDim.x) {
        const WorkItem it = b.lm_items[t];
        const Segment &seg = b.segs[it.segment];
        if (!seg.a.uncertainties)
            continue;
        switch (seg.model) {
        case kGaussian: covariance_fit<kGaussian>(seg.a, it.fit); break;
        case kLorentzian: covariance_fit<kLorentzian>(seg.a, it.fit); break;
        case kPseudoVoigt: covariance_fit<kPseudoVoigt>(seg.a, it.fit); break;
        default: covariance_fit<kTwoLorentzian>(seg.a, it.fit); break;
        }
    }
}

// ------------------------------------------------------------- synthetic --
// Counter-based uniform in (0, 1): SplitMix64 finaliser of (seed, stream, index).
__device__ __forceinline__ float uniform01(unsigned seed, unsigned long long stream, unsigned long long index) {
    unsigned long long z = (static_cast<unsigned long long>(seed) << 32) ^ (stream * 0x9e3779b97f4a7c15ull) ^ index;
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return (float(z >> 40) + 0.5f) * (1.0f / 16777216.0f);
}

template <int MODEL>
__global__ void __launch_bounds__(256) synthetic_kernel(int m, long long n, unsigned seed, float *x, float *y) {
    constexpr int P = Model<MODEL>::P;
    const long long total = n * m;
    const float dx = 20.0f / float(m > 1 ? m - 1 : 1);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long fit = t / m;
        const int j = int(t - fit * m);
        const float xj = j == m - 1 ? 10.0f : -10.0f + dx * float(j);
        if (fit == 0)
            x[j] = xj;
        auto u = [&](int k) { return uniform01(seed, (unsigned long long)fit, (unsigned long long)(k)); };
        const float amp = 0.5f + 4.5f * u(0);
        const float center = -6.0f + 12.0f * u(1);
        const float fwhm = 0.1f * __expf(u(2) * __logf(30.0f));
        float p[8] = {amp, center, fwhm, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if constexpr (MODEL == kGaussian)
            p[2] = fwhm / 2.354820045f;
        else if constexpr (MODEL == kLorentzian)
            p[2] = 0.5f * fwhm;
        else if constexpr (MODEL == kPseudoVoigt)
            p[3] = u(3);
        else {
            const float w2 = 0.2f * __expf(u(4) * __logf(10.0f));
            p[2] = 0.5f * fwhm;
            p[3] = amp * (0.1f + 0.9f * u(5));
            p[4] = center + (0.5f + 2.5f * u(6)) * 0.5f * (p[2] + w2);
            p[5] = w2;
        }
        const auto q = Model<MODEL>::prepare(p);
        float J[P];
        const float f = -Model<MODEL>::residual(q, xj, 0.0f, J);
        const float u1 = uniform01(seed, (unsigned long long)fit, 1000ull + 2ull * j);
        const float u2 = uniform01(seed, (unsigned long long)fit, 1001ull + 2ull * j);
        const float noise = sqrtf(-2.0f * __logf(u1)) * __cosf(6.283185307f * u2);
        y[t] = f + 0.01f * amp * noise;
    }
}

struct Grids {
    int device = -1;
    int guess = 0, lm[kLmClassTypes] = {}; // guess grid, LM grid per work-class type
};

using LmKernel = void (*)(BatchArgs);
#define BF_LM_FN(MODEL) batch_lm_kernel<MODEL, 8>, batch_lm_kernel<MODEL, 16>, batch_lm_kernel<MODEL, 32>
constexpr LmKernel kLmKernels[kLmClassTypes] = {BF_LM_FN(0), BF_LM_FN(1), BF_LM_FN(2), BF_LM_FN(3)};
#undef BF_LM_FN

// Grids for `sms` SMs' worth of blocks: blocks per SM resolved once per device
// (outside any stream capture: the first batch on a context launches directly).
cudaError_t grids_for(int sms, Grids &out) {
    constexpr int kDevices = 64;
    static Grids cache[kDevices];
    static std::mutex mutex;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
        return e;
    if (device < 0 || device >= kDevices)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mutex);
    auto scaled = [&](const Grids &per_sm) {
        out = per_sm;
        out.guess *= sms;
        for (int &l : out.lm)
            l *= sms;
    };
    if (cache[device].device == device) {
        scaled(cache[device]);
        return cudaSuccess;
    }
    int per_sm_guess = 0;
    e = batch_guess_blocks_per_sm(&per_sm_guess);
    Grids g;
    for (int k = 0; k < kLmClassTypes && e == cudaSuccess; ++k) {
        int per_sm = 0;
        e = cudaFuncSetAttribute(kLmKernels[k], cudaFuncAttributeMaxDynamicSharedMemorySize, kLmSmem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kLmKernels[k], kBatchLmBlock, kLmSmem);
        g.lm[k] = per_sm > 0 ? per_sm : 1;
    }
    if (e != cudaSuccess)
        return e;
    g.device = device;
    g.guess = per_sm_guess > 0 ? per_sm_guess : 1;
    cache[device] = g; // blocks per SM
    scaled(g);
    return cudaSuccess;
}

} // namespace

bool batch_guess_shape(int m, int *lanes, int *v) {
    const int n1 = pow2_at_least(edge_count(m));
    if (n1 <= 32) {
        *lanes = 8;
        *v = 4;
    } else if (n1 <= 128) {
        *lanes = 8;
        *v = 16;
    } else if (n1 <= 256) {
        *lanes = 16;
        *v = 16;
    } else if (n1 <= 512) {
        *lanes = 32;
        *v = 16;
    } else {
        *lanes = 32;
        *v = 0;
    }
    // The per-group share of the warp buffer holds the sort and the second-peak arrays.
    return n1 <= kBatchMaxSortWidth && second_peak_words(m, *lanes) <= kGuessWarpFloats / (32 / *lanes);
}

cudaError_t launch_synthetic(int model, int m, long long n, unsigned seed, float *x, float *y,
                             cudaStream_t stream) {
    const unsigned grid = 148u * 16u;
    switch (model) {
    case kGaussian: synthetic_kernel<kGaussian><<<grid, 256, 0, stream>>>(m, n, seed, x, y); break;
    case kLorentzian: synthetic_kernel<kLorentzian><<<grid, 256, 0, stream>>>(m, n, seed, x, y); break;
    case kPseudoVoigt: synthetic_kernel<kPseudoVoigt><<<grid, 256, 0, stream>>>(m, n, seed, x, y); break;
    default: synthetic_kernel<kTwoLorentzian><<<grid, 256, 0, stream>>>(m, n, seed, x, y); break;
    }
    return cudaGetLastError();
}

const void *batch_lm_function(int type) {
    return type >= 0 && type < kLmClassTypes ? reinterpret_cast<const void *>(kLmKernels[type]) : nullptr;
}

cudaError_t create_lm_fork(LmFork &f) {
    cudaError_t e = cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming);
    for (int s = 0; s < kLmStreams - 1 && e == cudaSuccess; ++s) {
        e = cudaStreamCreateWithFlags(&f.side[s], cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&f.join[s], cudaEventDisableTiming);
    }
    return e;
}

void release_lm_fork(LmFork &f) {
    for (int s = 0; s < kLmStreams - 1; ++s) {
        if (f.side[s]) {
            cudaStreamSynchronize(f.side[s]);
            cudaStreamDestroy(f.side[s]);
        }
        if (f.join[s])
            cudaEventDestroy(f.join[s]);
        f.side[s] = nullptr;
        f.join[s] = nullptr;
    }
    if (f.fork)
        cudaEventDestroy(f.fork);
    f.fork = nullptr;
}

cudaError_t launch_batch_pipeline(const BatchArgs &b, int sms, cudaStream_t stream, cudaEvent_t guessed,
                                  cudaEvent_t fitted, const LmFork *fork, uint32_t lm_types) {
    Grids grids;
    cudaError_t e = grids_for(sms, grids);
    if (e != cudaSuccess)
        return e;
    e = cudaMemsetAsync(b.counters, 0, 2 * kMaxClasses * sizeof(unsigned long long), stream);
    if (e != cudaSuccess)
        return e;
    batch_prepare_kernel<<<sms * 4, kBatchBlock, 0, stream>>>(b);
    launch_batch_guess(b, grids.guess, stream);
    if (guessed && (e = cudaEventRecord(guessed, stream)) != cudaSuccess)
        return e;
    // Heaviest types first (two-Lorentzian, then pseudo-Voigt, ...), dealt round-robin
    // over the streams.
    cudaStream_t lanes[kLmStreams] = {stream};
    const int streams = fork ? kLmStreams : 1;
    if (fork) {
        e = cudaEventRecord(fork->fork, stream);
        for (int s = 1; s < kLmStreams && e == cudaSuccess; ++s) {
            lanes[s] = fork->side[s - 1];
            e = cudaStreamWaitEvent(lanes[s], fork->fork, 0);
        }
        if (e != cudaSuccess)
            return e;
    }
    int dealt = 0;
    for (int k = kLmClassTypes - 1; k >= 0; --k)
        if (lm_types >> k & 1u)
            kLmKernels[k]<<<grids.lm[k], kBatchLmBlock, kLmSmem, lanes[dealt++ % streams]>>>(b);
    for (int s = 1; s < streams && e == cudaSuccess; ++s) {
        e = cudaEventRecord(fork->join[s - 1], lanes[s]);
        if (e == cudaSuccess)
            e = cudaStreamWaitEvent(stream, fork->join[s - 1], 0);
    }
    if (e != cudaSuccess)
        return e;
    if (fitted && (e = cudaEventRecord(fitted, stream)) != cudaSuccess)
        return e;
    batch_covariance_kernel<<<sms * 8, 128, 0, stream>>>(b);
    return cudaGetLastError();
}

} // namespace bf
