// Long spectra: fits whose spectrum does not fit the shared-memory layouts of the
// group kernels (guess_kernel, lm_kernel in bf_kernels.cu).  The reference fits any
// M (cpu::fit_batch, include/batchfit/cpu/batch.hpp:23-65; its Metal path moves long
// spectra to a whole-threadgroup-per-fit kernel, src/metal/cooperative.metal:16-34,
// 232-388, selected in include/batchfit/metal/batch.hpp:21-50).  Here:
//
// lm_cta_kernel: one CTA of kCtaThreads threads per fit.  x and the fit's y row are
//   read from global memory every pass; the rows of the CTAs resident on the GPU
//   (148 SMs x a few CTAs x 4 M bytes) stay in L2 between passes, so y comes from
//   HBM once.  Each thread accumulates a strided share of the points (the same
//   pass_sums code as the group kernels), each warp reduce-scatters its sums with
//   two-sum trees, and the warps' FP64 partials are added in a fixed order through
//   shared memory.  Every thread then runs the FP64 control redundantly
//   (lm_after_pass / lm_plan), so the CTA needs no broadcasts.
// guess_long_kernel: one warp per CTA per spectrum; initial_guess's general path
//   (V == 0) reads the row from global memory (the signal is computed on the fly,
//   not staged), with its sort and second-peak scratch in shared memory, or in a
//   caller-provided global buffer when that does not fit.
#include "bf_kernels.h"
#include "bf_lm.cuh"
#include "bf_xgrid.cuh"

namespace bf {

namespace {

constexpr int kCtaWarps = kCtaThreads / 32;

// 3- and 4-parameter models fit 128 registers (4 CTAs, 16 warps per SM); the
// two-Lorentzian takes 168 (3 CTAs), as in the group kernel.
template <int MODEL> struct CtaShape {
    static constexpr int min_blocks = MODEL == kTwoLorentzian ? 3 : 4;
};

template <int MODEL> struct CtaShared {
    static constexpr int K = Layout<MODEL>::K;
    double state[2 * K]; // accepted slot and pass slot (chi2, J^T r, lower J^T J)
    double warp_part[kCtaWarps][K];
    float warp_syy[kCtaWarps];
    XConst xc;
    long long fit;
};

// One pass of the CTA over its fit: per-thread sums, per-warp reduce-scatter, the
// warps' partials added in warp order.  Returns whether every sum is finite.
template <int MODEL, bool PAIRED_LOADS>
__device__ __forceinline__ bool lm_pass_cta(const float *x, const float *row, int m, const float *p,
                                            double *state, CtaShared<MODEL> &sh) {
    constexpr int K = Layout<MODEL>::K;
    constexpr int KP = reduce_slots(K, 32);
    const Group<32> g;
    float hi[KP], lo[KP];
    pass_sums<MODEL, kCtaThreads, PAIRED_LOADS>(int(threadIdx.x), x, row, m, p, hi, lo);
    double *mine = sh.warp_part[threadIdx.x / 32];
    bool finite = reduce_scatter_store<32, KP>(g, hi, lo, mine, K);
    finite = __syncthreads_and(finite);
    for (int t = int(threadIdx.x); t < K; t += kCtaThreads) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kCtaWarps; ++w)
            v += sh.warp_part[w][t];
        state[t] = v;
    }
    __syncthreads();
    return finite;
}

template <int MODEL>
__global__ void __launch_bounds__(kCtaThreads, CtaShape<MODEL>::min_blocks) lm_cta_kernel(FitArgs a) {
    constexpr int P = Model<MODEL>::P;
    constexpr int K = Layout<MODEL>::K;
    __shared__ CtaShared<MODEL> sh;
    const CtaGroup<kCtaThreads> cta;
    const int tid = int(threadIdx.x), warp = tid / 32;
    const int m = a.m;
    if (warp == 0) {
        const XConst xc = xconst_warp(a.x, m);
        if (tid == 0)
            sh.xc = xc;
    }
    __syncthreads();
    const XConst xc = sh.xc;
    const bool x_aligned = (reinterpret_cast<uintptr_t>(a.x) & 7u) == 0u;
    long long next_static = blockIdx.x;
    while (true) {
        if (tid == 0)
            sh.fit = a.work_counter ? (long long)atomicAdd(a.work_counter, 1ull) : next_static;
        next_static += gridDim.x;
        __syncthreads();
        const long long fit = sh.fit;
        __syncthreads();
        if (fit >= a.n)
            break;
        const float *row = a.y + fit * m;
        // Row checks (solver.hpp:223-226, 237-245) and sum(y^2) for the noise floor.
        const float y0 = __ldg(row);
        bool yfin = true, flat = true;
        float syy = 0.0f;
        for (int j = tid; j < m; j += kCtaThreads) {
            const float t = __ldg(row + j);
            yfin = yfin && isfinite(t);
            flat = flat && t == y0;
            syy = fmaf(t, t, syy);
        }
        yfin = __syncthreads_and(yfin);
        flat = __syncthreads_and(flat);
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1)
            syy += __shfl_xor_sync(0xffffffffu, syy, o);
        if ((tid & 31) == 0)
            sh.warp_syy[warp] = syy;
        __syncthreads();
        syy = 0.0f;
#pragma unroll
        for (int w = 0; w < kCtaWarps; ++w)
            syy += sh.warp_syy[w];
        LmState<MODEL> s;
        bool init_finite = true;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            s.p[k] = __ldg(a.p0 + fit * P + k);
            init_finite = init_finite && isfinite(s.p[k]);
        }
        if (!(a.options_ok && init_finite && xc.x_finite && yfin)) {
            // Preflight rejection (solver.hpp:205-226): parameters keep the initial values.
            s.status = kInvalid;
            s.iterations = 0;
            s.chi2 = __longlong_as_double(0x7ff8000000000000ll);
            write_fit<MODEL>(cta, a, fit, s);
            continue;
        }
        lm_begin<MODEL>(a, s);
        const bool paired = x_aligned && (reinterpret_cast<uintptr_t>(row) & 7u) == 0u;
        while (true) {
            double *slot = sh.state + (1 - s.cur) * K;
            const bool pass_finite = paired ? lm_pass_cta<MODEL, true>(a.x, row, m, s.t, slot, sh)
                                            : lm_pass_cta<MODEL, false>(a.x, row, m, s.t, slot, sh);
            bool done = lm_after_pass<MODEL>(cta, a, xc, flat, pass_finite, sh.state, s);
            if (!done)
                done = lm_plan<MODEL>(a, xc, double(syy), sh.state, s);
            if (done) {
                write_fit<MODEL>(cta, a, fit, s);
                if (a.uncertainties && s.status == kConverged)
                    write_information<MODEL>(cta, a, fit, sh.state + s.cur * K);
                __syncthreads();
                break;
            }
        }
    }
}

// initial_guess's scratch words for one spectrum of M points on 32 lanes (general
// path): the two sorted edge runs, or the second-peak search's arrays.
__host__ __device__ inline int long_guess_words(int m) {
    const int n1 = pow2_at_least(edge_count(m));
    const int peaks = second_peak_words(m, 32);
    return round_up(2 * n1 > peaks ? 2 * n1 : peaks, 4);
}

template <int MODEL>
__global__ void __launch_bounds__(32) guess_long_kernel(const float *x, const float *y, long long n, int m,
                                                      float *guesses, int32_t *guess_status, float *gscratch) {
    constexpr int P = Model<MODEL>::P;
    extern __shared__ __align__(16) float smem[];
    const Group<32> g;
    const XConst xc = xconst_warp(x, m);
    float *scratch = gscratch ? gscratch + (long long)blockIdx.x * long_guess_words(m) : smem;
    for (long long fit = blockIdx.x; fit < n; fit += gridDim.x) {
        const float *row = y + fit * m;
        const bool vec_ok = (m & 3) == 0 && (reinterpret_cast<uintptr_t>(row) & 15u) == 0u;
        bool yfin, flat;
        float syy;
        stage_row<32, false>(g, row, m, vec_ok, nullptr, yfin, flat, syy);
        float p[P];
        const int gs = initial_guess<MODEL, 32, 0>(g, xc, x, row, yfin, scratch, p);
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (int(g.lane) == k)
                guesses[fit * P + k] = p[k];
        if (g.lane == 0 && guess_status)
            guess_status[fit] = gs;
        g.sync();
    }
}

constexpr int kLongSmemLimit = 227 * 1024;
// CTAs per SM of the long guess when its scratch is in global memory (bounds the
// scratch buffer: grid x scratch words).
constexpr int kGlobalScratchCtasPerSm = 4;

bool long_guess_in_smem(int m) { return 4LL * long_guess_words(m) <= kLongSmemLimit; }

template <int MODEL>
cudaError_t launch_guess_long_typed(const float *x, const float *y, long long n, int m, float *guesses,
                                    int32_t *status, int sms, cudaStream_t stream, float *gscratch) {
    const bool in_smem = long_guess_in_smem(m);
    const int smem = in_smem ? 4 * long_guess_words(m) : 0;
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void *>(guess_long_kernel<MODEL>),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int per_sm = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, guess_long_kernel<MODEL>, 32, smem);
    if (e != cudaSuccess || n == 0)
        return e; // no fits: the kernel is loaded, nothing launched
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    if (!in_smem) {
        if (!gscratch)
            return cudaErrorInvalidValue;
        per_sm = per_sm < kGlobalScratchCtasPerSm ? per_sm : kGlobalScratchCtasPerSm;
    }
    long long grid = (long long)per_sm * sms;
    if (grid > n)
        grid = n;
    guess_long_kernel<MODEL><<<unsigned(grid), 32, smem, stream>>>(x, y, n, m, guesses, status,
                                                                   in_smem ? nullptr : gscratch);
    return cudaGetLastError();
}

template <int MODEL>
cudaError_t launch_lm_cta_typed(const FitArgs &a, int sms, cudaStream_t stream, LaunchInfo *info) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lm_cta_kernel<MODEL>, kCtaThreads, 0);
    if (e != cudaSuccess || a.n == 0)
        return e;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    long long grid = (long long)per_sm * sms;
    if (grid > a.n)
        grid = a.n;
    lm_cta_kernel<MODEL><<<unsigned(grid), kCtaThreads, 0, stream>>>(a);
    if (info)
        *info = LaunchInfo{int(grid), kCtaThreads, 0, per_sm, kCtaThreads};
    return cudaGetLastError();
}

} // namespace

size_t long_guess_scratch_bytes(int m, int sms) {
    if (long_guess_in_smem(m))
        return 0;
    return size_t(kGlobalScratchCtasPerSm) * size_t(sms) * size_t(long_guess_words(m)) * sizeof(float);
}

int long_guess_smem_max_points() {
    int lo = 1, hi = kMaxPoints;
    while (lo < hi) {
        const int mid = lo + (hi - lo + 1) / 2;
        if (long_guess_in_smem(mid))
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

cudaError_t launch_guess_long(int model, const float *x, const float *y, long long n, int m, float *guesses,
                              int32_t *status, int sms, cudaStream_t stream, float *gscratch) {
    switch (model) {
    case kGaussian: return launch_guess_long_typed<kGaussian>(x, y, n, m, guesses, status, sms, stream, gscratch);
    case kLorentzian: return launch_guess_long_typed<kLorentzian>(x, y, n, m, guesses, status, sms, stream, gscratch);
    case kPseudoVoigt:
        return launch_guess_long_typed<kPseudoVoigt>(x, y, n, m, guesses, status, sms, stream, gscratch);
    case kTwoLorentzian:
        return launch_guess_long_typed<kTwoLorentzian>(x, y, n, m, guesses, status, sms, stream, gscratch);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_lm_cta(int model, const FitArgs &a, int sms, cudaStream_t stream, LaunchInfo *info) {
    switch (model) {
    case kGaussian: return launch_lm_cta_typed<kGaussian>(a, sms, stream, info);
    case kLorentzian: return launch_lm_cta_typed<kLorentzian>(a, sms, stream, info);
    case kPseudoVoigt: return launch_lm_cta_typed<kPseudoVoigt>(a, sms, stream, info);
    case kTwoLorentzian: return launch_lm_cta_typed<kTwoLorentzian>(a, sms, stream, info);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace bf
