// Fit kernels: one thread group (8, 16 or 32 lanes) per spectrum.
//
// guess_kernel: the data-only initial guess per spectrum (spectrum staged in
//   shared memory, group-parallel searches), written to a [N,P] buffer.
// lm_kernel: persistent bounded LM in rounds.  Every round each group runs exactly
//   one fused pass for its fit -- the initial cost/linearisation of a newly
//   claimed fit or the trial of an ongoing one -- then its FP64 control.  A group
//   whose fit finished claims the next one (atomic work counter) at the start of
//   the following round, so the groups of a warp stay in the same code (the pass)
//   instead of drifting through different phases.
//
// Per CTA the shared x grid is staged in shared memory once and its derived
// constants computed there.  Per group the fit-major y row is staged with 128-bit
// streaming loads; group buffers are offset by G banks so the groups of a warp
// read disjoint banks.
#include "bf_kernels.h"
#include "bf_lm.cuh"

namespace bf {

// Guess kernel CTA shape per register-sort width V: up to 8 values per lane the
// guess fits in 96 registers, so 128-thread CTAs, 5 per SM (20 warps); wider sorts
// need 128 registers: 256 threads, 2 per SM.
__host__ __device__ constexpr int guess_threads(int v) { return v > 0 && v <= 8 ? 128 : 256; }
template <int V> struct GuessShapeCfg {
    static constexpr int threads = guess_threads(V);
    static constexpr int min_blocks = V > 0 && V <= 8 ? 5 : 2;
};
// LM kernel CTA shape per model and group width.  The 3- and 4-parameter paired
// passes need 128 registers a thread: 128-thread CTAs, 4 per SM (16 warps).  At 5
// per SM (96 registers) the pseudo-Voigt spills 82 bytes and runs 5-20% slower, but
// the Lorentzian and Gaussian at 8 lanes fit (95-96 registers, 0-4 bytes) and run
// 2-7% faster at M = 256 and 512, where the lane rule uses 8 lanes.  The
// two-Lorentzian state (8 parameters, 36 J^T J sums, an 8x8 FP64 Cholesky) spills
// heavily at 128 registers; 128-thread CTAs, 3 per SM, allow 168 (12 warps per SM,
// little spilling) -- measured 5% faster on B200 than 256 threads, 2 per SM.
template <int MODEL, int G = 8> struct LmShape {
    static constexpr int threads = 128;
    static constexpr int min_blocks =
        MODEL == kTwoLorentzian ? 3 : (MODEL != kPseudoVoigt && G == 8) ? 5 : 4;
};

// Per-group shared memory, in 4-byte words, padded so that consecutive groups of a
// warp start G banks apart.
__host__ __device__ inline int bank_staggered(int words, int lanes) { return round_up(words, 32) + (lanes % 32); }

// The LM pass reads its row as 8-byte pairs, which a warp serves in two phases of 16
// lanes: groups of 8 lanes start 16 banks apart so that the two groups of a phase
// read disjoint banks (wider groups fill a phase alone).
template <int MODEL> __host__ __device__ inline int lm_group_words(int m, int lanes) {
    return round_up(round_up(m, 4) + 4 * Layout<MODEL>::K, 32) + (2 * lanes) % 32; // y row + 2 FP64 state slots
}
__host__ __device__ inline int guess_group_words(int m, int lanes, int v) {
    const int n1 = pow2_at_least(edge_count(m));
    const int sorted = n1 > lanes * v ? n1 : lanes * v;
    const int peaks = second_peak_words(m, lanes);
    // y row + scratch: the sorted edge runs, later the second-peak search's arrays
    return bank_staggered(round_up(m, 4) + (2 * sorted > peaks ? 2 * sorted : peaks), lanes);
}
__host__ __device__ inline int x_words(int m) { return round_up(m, 4); }

template <int MODEL, int G> int lm_smem_bytes(int m) {
    return 4 * (x_words(m) + (LmShape<MODEL>::threads / G) * lm_group_words<MODEL>(m, G));
}
template <int G, int V> int guess_smem_bytes(int m) {
    return 4 * (x_words(m) + (GuessShapeCfg<V>::threads / G) * guess_group_words(m, G, V));
}

// CTA prologue: stage x and derive the grid constants (solver.hpp:58-69,223-239;
// initial_guess.hpp:131-153).  Called by every thread of the block.
__device__ void cta_prologue(const float *x, int m, float *xs, XConst &xc) {
    __shared__ unsigned int min_abs_bits, min_diff_bits;
    const int tid = threadIdx.x;
    if (tid == 0) {
        min_abs_bits = 0x7f800000u;
        min_diff_bits = 0x7f800000u;
    }
    for (int j = tid; j < m; j += blockDim.x)
        xs[j] = x[j];
    __syncthreads();
    bool fin = true, up = true, down = true, strict = true, varied = false;
    for (int j = tid; j < m; j += blockDim.x) {
        const float v = xs[j];
        fin = fin && isfinite(v);
        varied = varied || v != xs[0];
        if (j > 0) {
            const float d = v - xs[j - 1];
            up = up && d >= 0.0f;
            down = down && d <= 0.0f;
            if (d != 0.0f && isfinite(d))
                atomicMin(&min_abs_bits, __float_as_uint(fabsf(d)));
            strict = strict && v > xs[j - 1];
            if (d > 0.0f)
                atomicMin(&min_diff_bits, __float_as_uint(d));
        }
    }
    fin = __syncthreads_and(fin);
    up = __syncthreads_and(up);
    down = __syncthreads_and(down);
    strict = __syncthreads_and(strict);
    varied = __syncthreads_or(varied);
    if (tid == 0) {
        xc.m = m;
        xc.x_finite = fin;
        xc.varied_x = varied;
        const float spacing = __uint_as_float(min_abs_bits);
        xc.spacing = (up || down) && isfinite(spacing) ? spacing : 0.0f;
        const int count = edge_count(m);
        xc.count = count;
        xc.n1 = pow2_at_least(count);
        xc.guess_ok = m >= 5 && fin && strict && isfinite(rsub(xs[m - 1], xs[0]));
        xc.guess_spacing = __uint_as_float(min_diff_bits);
        xc.left_x = midpoint_rn(xs[(count - 1) / 2], xs[count / 2]);
        xc.right_x = midpoint_rn(xs[m - count + (count - 1) / 2], xs[m - count + count / 2]);
    }
    __syncthreads();
}

// ------------------------------------------------------------ guess kernel --
// G lanes per spectrum; V edge values per lane sorted in registers (V == 0: the
// shared-memory sorting path for very long spectra).
template <int MODEL, int G, int V>
__global__ void __launch_bounds__(GuessShapeCfg<V>::threads, GuessShapeCfg<V>::min_blocks) guess_kernel(const float *x, const float *y, long long n,
                                                                   int m, float *guesses, int32_t *guess_status,
                                                                   int y_half) {
    constexpr int P = Model<MODEL>::P;
    constexpr int kGroups = GuessShapeCfg<V>::threads / G;
    extern __shared__ __align__(16) float smem[];
    __shared__ XConst xc;
    float *xs = smem;
    cta_prologue(x, m, xs, xc);
    const XConst cx = xc;
    const Group<G> g;
    const int gid = threadIdx.x / G;
    float *ys = smem + x_words(m) + gid * guess_group_words(m, G, V);
    float *scratch = ys + round_up(m, 4);
    const bool vec_ok = rows_vectorisable(y, m, y_half);
    for (long long fit = (long long)blockIdx.x * kGroups + gid; fit < n; fit += (long long)gridDim.x * kGroups) {
        bool yfin, flat;
        float syy;
        stage_fit_row<G, false>(g, y, y_half, fit, m, vec_ok, ys, yfin, flat, syy); // the guess needs only yfin
        float p[P];
        const int gs = initial_guess<MODEL, G, V, true>(g, cx, xs, ys, yfin, scratch, p);
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (int(g.lane) == k)
                guesses[fit * P + k] = p[k];
        if (g.lane == 0 && guess_status)
            guess_status[fit] = gs;
        g.sync();
    }
}

// --------------------------------------------------------------- LM kernel --
template <int MODEL, int G>
__global__ void __launch_bounds__(LmShape<MODEL, G>::threads, LmShape<MODEL, G>::min_blocks) lm_kernel(FitArgs a) {
    constexpr int P = Model<MODEL>::P;
    constexpr int kGroups = LmShape<MODEL>::threads / G;
    extern __shared__ __align__(16) float smem[];
    __shared__ XConst xc;
    const int m = a.m;
    float *xs = smem;
    cta_prologue(a.x, m, xs, xc);
    const XConst cx = xc;
    const Group<G> g;
    const int gid = threadIdx.x / G;
    float *ys = smem + x_words(m) + gid * lm_group_words<MODEL>(m, G);
    double *state = reinterpret_cast<double *>(ys + round_up(m, 4));
    const bool vec_ok = rows_vectorisable(a.y, m, a.y_half);
    long long next_static = (long long)blockIdx.x * kGroups + gid;
    LmState<MODEL> s;
    long long fit = -1;
    bool flat = false;
    float syy = 0.0f;
    while (true) {
        if (fit < 0) {
            // Intake: claim fits until one needs a pass or the queue is empty.
            while (true) {
                long long f;
                if (a.work_counter) {
                    unsigned long long t = 0;
                    if (g.lane == 0)
                        t = atomicAdd(a.work_counter, 1ull);
                    f = (long long)g.bcast(t, 0);
                } else {
                    f = next_static;
                    next_static += (long long)gridDim.x * kGroups;
                }
                if (f >= a.n)
                    break;
                bool yfin;
                stage_fit_row(g, a.y, a.y_half, f, m, vec_ok, ys, yfin, flat, syy);
                bool init_finite = true;
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    s.p[k] = __ldg(a.p0 + f * P + k);
                    init_finite = init_finite && isfinite(s.p[k]);
                }
                if (a.options_ok && init_finite && cx.x_finite && yfin) {
                    lm_begin<MODEL>(a, s);
                    fit = f;
                    break;
                }
                // Preflight rejection (solver.hpp:205-226): parameters keep the initial values.
                s.status = kInvalid;
                s.iterations = 0;
                s.chi2 = __longlong_as_double(0x7ff8000000000000ll);
                write_fit<MODEL>(g, a, f, s);
            }
            if (fit < 0)
                break;
        }
        const bool pass_finite = lm_pass<MODEL, G, true>(g, xs, ys, m, s.t, state + (1 - s.cur) * Layout<MODEL>::K);
        bool done = lm_after_pass<MODEL>(g, a, cx, flat, pass_finite, state, s);
        if (!done)
            done = lm_plan<MODEL>(a, cx, double(syy), state, s);
        if (done) {
            write_fit<MODEL>(g, a, fit, s);
            if (a.uncertainties && s.status == kConverged)
                write_information<MODEL>(g, a, fit, state + s.cur * Layout<MODEL>::K);
            g.sync();
            fit = -1;
        }
    }
}

// ------------------------------------------------------- covariance kernel --
// One thread per fit: reads the status, parameters, chi2 and the information
// matrix the LM kernel left in the covariance output; writes covariance, standard
// errors and the uncertainty status.
constexpr int kCovBlock = 128;

template <int MODEL> __global__ void __launch_bounds__(kCovBlock) covariance_kernel(FitArgs a) {
    const long long fit = (long long)blockIdx.x * kCovBlock + threadIdx.x;
    if (fit < a.n)
        covariance_fit<MODEL>(a, fit);
}

// ------------------------------------------------ roofline microbenchmarks --
// Throughput of the pipes the fit kernels are bound by, measured on the device the
// fits run on: 8 independent dependency chains per thread, enough warps to cover
// the pipe latency.  `sink` only keeps the chains alive.
constexpr int kPeakChains = 8;

__global__ void __launch_bounds__(256) peak_ffma_kernel(float *sink, int iters) {
    float a[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k)
        a[k] = float(threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kPeakChains; ++k)
            a[k] = fmaf(a[k], 0.999999f, 1e-7f);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k)
        s += a[k];
    if (s == -1.0f)
        sink[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) peak_dfma_kernel(double *sink, int iters) {
    double a[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k)
        a[k] = double(threadIdx.x + k) * 1e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kPeakChains; ++k)
            a[k] = fma(a[k], 0.999999, 1e-7);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k)
        s += a[k];
    if (s == -1.0)
        sink[blockIdx.x] = s;
}

template <bool EX2> __global__ void __launch_bounds__(256) peak_mufu_kernel(float *sink, int iters) {
    float a[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k)
        a[k] = 0.5f + float(threadIdx.x + k) * 1e-4f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kPeakChains; ++k)
            a[k] = EX2 ? ex2_approx(-a[k]) : rcp_approx(a[k] + 1.0f);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k)
        s += a[k];
    if (s == -1.0f)
        sink[blockIdx.x] = s;
}

template <class F> static cudaError_t time_best(F launch, cudaStream_t s, float &best_ms) {
    cudaEvent_t e0, e1;
    cudaError_t e = cudaEventCreate(&e0);
    if (e != cudaSuccess)
        return e;
    e = cudaEventCreate(&e1);
    best_ms = 1e30f;
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
        cudaEventRecord(e0, s);
        launch();
        cudaEventRecord(e1, s);
        e = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best_ms)
            best_ms = ms; // first run is a warm-up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

cudaError_t measure_peaks(int sms, cudaStream_t s, PeakRates *out) {
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    void *sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, size_t(blocks) * sizeof(double));
    if (e != cudaSuccess)
        return e;
    const double lanes = double(blocks) * threads * kPeakChains * iters;
    float ms = 0.0f;
    e = time_best([&] { peak_ffma_kernel<<<blocks, threads, 0, s>>>(static_cast<float *>(sink), iters); }, s, ms);
    if (e == cudaSuccess)
        out->fp32_tflops = 2.0 * lanes / (ms * 1e-3) / 1e12;
    if (e == cudaSuccess)
        e = time_best([&] { peak_dfma_kernel<<<blocks, threads, 0, s>>>(static_cast<double *>(sink), iters / 4); },
                      s, ms);
    if (e == cudaSuccess)
        out->fp64_tflops = 2.0 * lanes / 4 / (ms * 1e-3) / 1e12;
    if (e == cudaSuccess)
        e = time_best([&] { peak_mufu_kernel<true><<<blocks, threads, 0, s>>>(static_cast<float *>(sink), iters / 4); },
                      s, ms);
    if (e == cudaSuccess)
        out->mufu_ex2_gops = lanes / 4 / (ms * 1e-3) / 1e9;
    if (e == cudaSuccess)
        e = time_best(
            [&] { peak_mufu_kernel<false><<<blocks, threads, 0, s>>>(static_cast<float *>(sink), iters / 4); }, s, ms);
    if (e == cudaSuccess)
        out->mufu_rcp_gops = lanes / 4 / (ms * 1e-3) / 1e9;
    cudaFree(sink);
    return e;
}

// ------------------------------------------------------------ host side --
template <class K> static cudaError_t grid_for(K kernel, int block, int smem, long long groups_needed,
                                               int groups_per_cta, int sms, int &grid, int &per_sm) {
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void *>(kernel),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess)
        return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem);
    if (e != cudaSuccess)
        return e;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    long long want = (groups_needed + groups_per_cta - 1) / groups_per_cta;
    long long g = (long long)per_sm * sms;
    if (want < g)
        g = want;
    grid = int(g < 1 ? 1 : g);
    return cudaSuccess;
}

template <int MODEL, int G>
static cudaError_t launch_lm_typed(const FitArgs &a, int sms, cudaStream_t stream, LaunchInfo *info) {
    const int smem = lm_smem_bytes<MODEL, G>(a.m);
    int grid = 0, per_sm = 0;
    constexpr int kThreads = LmShape<MODEL>::threads;
    cudaError_t e = grid_for(lm_kernel<MODEL, G>, kThreads, smem, a.n, kThreads / G, sms, grid, per_sm);
    if (e != cudaSuccess || a.n == 0)
        return e; // no fits: setting the attributes above has loaded the kernel
    lm_kernel<MODEL, G><<<grid, kThreads, smem, stream>>>(a);
    if (info)
        *info = LaunchInfo{grid, kThreads, smem, per_sm, G};
    return cudaGetLastError();
}

template <int MODEL> static cudaError_t launch_covariance_typed(const FitArgs &a, cudaStream_t stream) {
    if (a.n == 0) {
        cudaFuncAttributes attr; // loads the kernel
        return cudaFuncGetAttributes(&attr, covariance_kernel<MODEL>);
    }
    covariance_kernel<MODEL><<<unsigned((a.n + kCovBlock - 1) / kCovBlock), kCovBlock, 0, stream>>>(a);
    return cudaGetLastError();
}

template <int MODEL, int G, int V>
static cudaError_t launch_guess_typed(const float *x, const float *y, long long n, int m, float *guesses,
                                      int32_t *status, int sms, cudaStream_t stream, int y_half) {
    const int smem = guess_smem_bytes<G, V>(m);
    int grid = 0, per_sm = 0;
    constexpr int kThreads = GuessShapeCfg<V>::threads;
    cudaError_t e = grid_for(guess_kernel<MODEL, G, V>, kThreads, smem, n, kThreads / G, sms, grid, per_sm);
    if (e != cudaSuccess || n == 0)
        return e; // no fits: the kernel is loaded (its attributes set), nothing launched
    guess_kernel<MODEL, G, V><<<grid, kThreads, smem, stream>>>(x, y, n, m, guesses, status, y_half);
    return cudaGetLastError();
}

// Group width and register-sort width of the guess for spectra of M points: the
// edge runs hold max(1, M/10) values each.
struct GuessShape {
    int lanes, v;
};
// Every staged row takes shared memory, so from M=640 on the fits in flight per
// SM are bounded by it: wider groups (up to 32 lanes) with at most 8 sort values a
// lane keep 128-thread CTAs and split each fit over more lanes.  Measured on B200
// (same results for every shape): pseudo-Voigt M=1024 8x16 1.18 ms -> 16x8 0.99 ms
// per 262,144 fits; M=2048 16x16 1.26 ms -> 32x8 1.01 ms per 131,072 fits;
// two-Lorentzian M=1024 7.78 -> 6.08 ms per 262,144 fits.
__host__ __device__ inline GuessShape guess_shape(int m) {
    const int n1 = pow2_at_least(edge_count(m));
    if (n1 <= 64)
        return {8, n1 / 8 > 1 ? n1 / 8 : 1};
    if (n1 <= 128)
        return {16, 8};
    if (n1 <= 256)
        return {32, 8};
    if (n1 <= 512)
        return {32, 16};
    return {32, 0};
}

template <int MODEL>
static cudaError_t launch_lm_model(const FitArgs &a, int lanes, int sms, cudaStream_t s, LaunchInfo *info,
                                   cudaEvent_t lm_done) {
    cudaError_t e;
    switch (lanes) {
    case 8: e = launch_lm_typed<MODEL, 8>(a, sms, s, info); break;
    case 16: e = launch_lm_typed<MODEL, 16>(a, sms, s, info); break;
    case 32: e = launch_lm_typed<MODEL, 32>(a, sms, s, info); break;
    case kCtaLanes: e = launch_lm_cta(MODEL, a, sms, s, info); break;
    default: return cudaErrorInvalidValue;
    }
    if (e == cudaSuccess && lm_done)
        e = cudaEventRecord(lm_done, s);
    if (e != cudaSuccess || !a.uncertainties)
        return e;
    return launch_covariance_typed<MODEL>(a, s);
}

template <int MODEL>
static cudaError_t launch_guess_model(const float *x, const float *y, long long n, int m, float *guesses,
                                      int32_t *status, int sms, cudaStream_t s, int y_half) {
    const GuessShape gs = guess_shape(m);
    switch (gs.lanes * 100 + gs.v) {
    case 801: return launch_guess_typed<MODEL, 8, 1>(x, y, n, m, guesses, status, sms, s, y_half);
    case 802: return launch_guess_typed<MODEL, 8, 2>(x, y, n, m, guesses, status, sms, s, y_half);
    case 804: return launch_guess_typed<MODEL, 8, 4>(x, y, n, m, guesses, status, sms, s, y_half);
    case 808: return launch_guess_typed<MODEL, 8, 8>(x, y, n, m, guesses, status, sms, s, y_half);
    case 1608: return launch_guess_typed<MODEL, 16, 8>(x, y, n, m, guesses, status, sms, s, y_half);
    case 3208: return launch_guess_typed<MODEL, 32, 8>(x, y, n, m, guesses, status, sms, s, y_half);
    case 3216: return launch_guess_typed<MODEL, 32, 16>(x, y, n, m, guesses, status, sms, s, y_half);
    default: return launch_guess_typed<MODEL, 32, 0>(x, y, n, m, guesses, status, sms, s, y_half);
    }
}

cudaError_t launch_fit(int model, int lanes, const FitArgs &a, int sms, cudaStream_t s, LaunchInfo *info,
                       cudaEvent_t lm_done) {
    switch (model) {
    case kGaussian: return launch_lm_model<kGaussian>(a, lanes, sms, s, info, lm_done);
    case kLorentzian: return launch_lm_model<kLorentzian>(a, lanes, sms, s, info, lm_done);
    case kPseudoVoigt: return launch_lm_model<kPseudoVoigt>(a, lanes, sms, s, info, lm_done);
    case kTwoLorentzian: return launch_lm_model<kTwoLorentzian>(a, lanes, sms, s, info, lm_done);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_guess(int model, const float *x, const float *y, long long n, int m, float *guesses,
                         int32_t *status, int sms, cudaStream_t s, int y_half, float *gscratch) {
    if (m > group_guess_max_points()) {
        if (y_half)
            return cudaErrorInvalidValue; // long spectra take float32 y
        return launch_guess_long(model, x, y, n, m, guesses, status, sms, s, gscratch);
    }
    switch (model) {
    case kGaussian: return launch_guess_model<kGaussian>(x, y, n, m, guesses, status, sms, s, y_half);
    case kLorentzian: return launch_guess_model<kLorentzian>(x, y, n, m, guesses, status, sms, s, y_half);
    case kPseudoVoigt: return launch_guess_model<kPseudoVoigt>(x, y, n, m, guesses, status, sms, s, y_half);
    case kTwoLorentzian: return launch_guess_model<kTwoLorentzian>(x, y, n, m, guesses, status, sms, s, y_half);
    default: return cudaErrorInvalidValue;
    }
}

int group_smem_bytes(int model, int lanes, int m) {
    switch (model * 100 + lanes) {
    case 8: return lm_smem_bytes<0, 8>(m);
    case 16: return lm_smem_bytes<0, 16>(m);
    case 32: return lm_smem_bytes<0, 32>(m);
    case 108: return lm_smem_bytes<1, 8>(m);
    case 116: return lm_smem_bytes<1, 16>(m);
    case 132: return lm_smem_bytes<1, 32>(m);
    case 208: return lm_smem_bytes<2, 8>(m);
    case 216: return lm_smem_bytes<2, 16>(m);
    case 232: return lm_smem_bytes<2, 32>(m);
    case 308: return lm_smem_bytes<3, 8>(m);
    case 316: return lm_smem_bytes<3, 16>(m);
    default: return lm_smem_bytes<3, 32>(m);
    }
}

static int guess_smem(int m) {
    const GuessShape s = guess_shape(m);
    return 4 * (x_words(m) + (guess_threads(s.v) / s.lanes) * guess_group_words(m, s.lanes, s.v));
}

// Largest M with fits(M) (monotone) up to kMaxPoints.
template <class F> static int largest_m(F fits) {
    int lo = 1, hi = kMaxPoints;
    while (lo < hi) {
        const int mid = lo + (hi - lo + 1) / 2;
        if (fits(mid))
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

constexpr int kSmemLimit = 227 * 1024;

int group_lm_max_points(int model) {
    return largest_m([model](int m) { return group_smem_bytes(model, 32, m) <= kSmemLimit; });
}

int group_guess_max_points() {
    static const int limit = largest_m([](int m) { return guess_smem(m) <= kSmemLimit; });
    return limit;
}

} // namespace bf
