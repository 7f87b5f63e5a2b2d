// Persistent fit kernels: one thread group (8, 16 or 32 lanes) per spectrum.
//
// Per CTA: the shared x grid is staged in shared memory once and its derived
// constants (finiteness, monotone spacing, guess edge abscissae) computed there.
// Per group: claim a fit (atomic work counter), stage its fit-major y row in
// shared memory with 128-bit streaming loads, run the data-only guess when no
// initial values are given, run bounded LM, and write the outputs.
#include "bf_kernels.h"
#include "bf_lm.cuh"

#include <cstdio>

namespace bf {

constexpr int kBlock = 256;
constexpr int kMinBlocks = 2;

__host__ __device__ inline int round_up(int v, int a) { return (v + a - 1) / a * a; }
__host__ __device__ inline int edge_count(int m) { return m / 10 > 1 ? m / 10 : 1; }
__host__ __device__ inline int pow2_at_least(int v) {
    int p = 1;
    while (p < v)
        p <<= 1;
    return p;
}

template <int MODEL> __host__ __device__ inline int group_smem_bytes(int m) {
    const int n1 = pow2_at_least(edge_count(m));
    int bytes = 4 * round_up(m, 4) + 4 * 2 * n1;
    bytes = round_up(bytes, 16);
    bytes += 2 * Layout<MODEL>::K * 8;
    return round_up(bytes, 16);
}

template <int MODEL, int G> int kernel_smem_bytes(int m) {
    return 4 * round_up(m, 4) + (kBlock / G) * group_smem_bytes<MODEL>(m);
}

template <int MODEL, int G> __global__ void __launch_bounds__(kBlock, kMinBlocks) fit_kernel(FitArgs a, GuessArgs ga) {
    constexpr int P = Model<MODEL>::P;
    constexpr int kGroups = kBlock / G;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ XConst xc;
    __shared__ unsigned int min_abs_bits, min_diff_bits;
    const int m = a.m;
    float *xs = reinterpret_cast<float *>(smem);
    const int tid = threadIdx.x;

    // ---- CTA prologue: stage x and derive the grid constants. ----
    if (tid == 0) {
        min_abs_bits = 0x7f800000u;
        min_diff_bits = 0x7f800000u;
    }
    for (int j = tid; j < m; j += kBlock)
        xs[j] = a.x[j];
    __syncthreads();
    bool fin = true, up = true, down = true, strict = true, varied = false;
    for (int j = tid; j < m; j += kBlock) {
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
    const XConst cx = xc;

    // ---- per-group buffers ----
    const Group<G> g;
    const int gid = tid / G;
    unsigned char *gbase = smem + 4 * round_up(m, 4) + gid * group_smem_bytes<MODEL>(m);
    float *ys = reinterpret_cast<float *>(gbase);
    float *scratch = ys + round_up(m, 4);
    double *state = reinterpret_cast<double *>(gbase + round_up(4 * round_up(m, 4) + 8 * cx.n1, 16));
    const bool vec_ok = (m & 3) == 0 && (reinterpret_cast<uintptr_t>(a.y) & 15) == 0;

    long long next_static = (long long)blockIdx.x * kGroups + gid;
    while (true) {
        long long fit;
        if (a.work_counter) {
            unsigned long long t = 0;
            if (g.lane == 0)
                t = atomicAdd(a.work_counter, 1ull);
            fit = (long long)g.bcast(t, 0);
        } else {
            fit = next_static;
            next_static += (long long)gridDim.x * kGroups;
        }
        if (fit >= a.n)
            break;

        // ---- stage y (fit-major row) ----
        const float *row = a.y + fit * (long long)m;
        const float y0 = __ldg(row);
        bool yfin = true, flat = true;
        float syy = 0.0f;
        if (vec_ok) {
            const float4 *row4 = reinterpret_cast<const float4 *>(row);
            for (int v = int(g.lane); v < m / 4; v += G) {
                const float4 t = __ldcs(row4 + v);
                reinterpret_cast<float4 *>(ys)[v] = t;
                yfin = yfin && isfinite(t.x) && isfinite(t.y) && isfinite(t.z) && isfinite(t.w);
                flat = flat && t.x == y0 && t.y == y0 && t.z == y0 && t.w == y0;
                syy = fmaf(t.x, t.x, fmaf(t.y, t.y, fmaf(t.z, t.z, fmaf(t.w, t.w, syy))));
            }
        } else {
            for (int j = int(g.lane); j < m; j += G) {
                const float t = __ldcs(row + j);
                ys[j] = t;
                yfin = yfin && isfinite(t);
                flat = flat && t == y0;
                syy = fmaf(t, t, syy);
            }
        }
        yfin = g.all(yfin);
        flat = g.all(flat);
#pragma unroll
        for (int o = G / 2; o >= 1; o >>= 1)
            syy += g.xor_(syy, o);
        g.sync();

        // ---- initial values ----
        float p[P];
        if (a.p0) {
#pragma unroll
            for (int k = 0; k < P; ++k)
                p[k] = __ldg(a.p0 + fit * P + k);
        } else {
            const int gs = initial_guess<MODEL, G>(g, cx, xs, ys, yfin, scratch, p);
            if (ga.guesses) {
#pragma unroll
                for (int k = 0; k < P; ++k)
                    if (int(g.lane) == k)
                        ga.guesses[fit * P + k] = p[k];
                if (g.lane == 0 && ga.guess_status)
                    ga.guess_status[fit] = gs;
            }
        }
        if (ga.guess_only) {
            g.sync();
            continue;
        }

        // ---- LM ----
        int slot = 0;
        const FitOutcome r = lm_solve<MODEL, G>(g, a, cx, xs, ys, yfin, flat, double(syy), p, state, slot);
        const float chi2f = float(r.chi2);
#pragma unroll
        for (int k = 0; k < P; ++k)
            if (int(g.lane) == k)
                a.params[fit * P + k] = p[k];
        if (g.lane == 0) {
            a.status[fit] = r.status;
            a.iterations[fit] = r.iterations;
            a.chi2[fit] = chi2f;
        }
        if (a.uncertainties) {
            const int us = lm_uncertainty<MODEL, G>(g, a, cx, p, r.status, chi2f, state,
                                                    state + slot * Layout<MODEL>::K, a.policy == kPolicyParity,
                                                    a.covariance + fit * P * P, a.stderr_out + fit * P);
            if (g.lane == 0)
                a.ustatus[fit] = us;
        }
        g.sync();
    }
}

// ------------------------------------------------------------ host side --
template <int MODEL, int G> static const void *kernel_ptr() {
    return reinterpret_cast<const void *>(&fit_kernel<MODEL, G>);
}

template <int MODEL, int G>
static cudaError_t launch_typed(const FitArgs &a, const GuessArgs &ga, int sms, cudaStream_t stream,
                                LaunchInfo *info) {
    const int smem = kernel_smem_bytes<MODEL, G>(a.m);
    cudaError_t e = cudaFuncSetAttribute(kernel_ptr<MODEL, G>(), cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess)
        return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fit_kernel<MODEL, G>, kBlock, smem);
    if (e != cudaSuccess)
        return e;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    constexpr int groups = kBlock / G;
    long long want = (a.n + groups - 1) / groups;
    long long grid = (long long)per_sm * sms;
    if (want < grid)
        grid = want;
    if (grid < 1)
        grid = 1;
    fit_kernel<MODEL, G><<<unsigned(grid), kBlock, smem, stream>>>(a, ga);
    if (info) {
        info->grid = int(grid);
        info->block = kBlock;
        info->smem = smem;
        info->blocks_per_sm = per_sm;
        info->group_lanes = G;
    }
    return cudaGetLastError();
}

template <int MODEL>
static cudaError_t launch_model(const FitArgs &a, const GuessArgs &ga, int lanes, int sms, cudaStream_t s,
                                LaunchInfo *info) {
    switch (lanes) {
    case 8:
        return launch_typed<MODEL, 8>(a, ga, sms, s, info);
    case 16:
        return launch_typed<MODEL, 16>(a, ga, sms, s, info);
    default:
        return launch_typed<MODEL, 32>(a, ga, sms, s, info);
    }
}

int max_points(int model) {
    // Largest M whose per-CTA layout (x plus one 32-lane group... kBlock/32 groups) fits
    // the 227 KB opt-in shared memory of one CTA.
    const int limit = 227 * 1024;
    int lo = 1, hi = 1 << 20;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        int bytes = 0;
        switch (model) {
        case 0: bytes = kernel_smem_bytes<0, 32>(mid); break;
        case 1: bytes = kernel_smem_bytes<1, 32>(mid); break;
        case 2: bytes = kernel_smem_bytes<2, 32>(mid); break;
        default: bytes = kernel_smem_bytes<3, 32>(mid); break;
        }
        if (bytes <= limit)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

int smem_bytes(int model, int lanes, int m) {
    switch (model * 100 + lanes) {
    case 8: return kernel_smem_bytes<0, 8>(m);
    case 16: return kernel_smem_bytes<0, 16>(m);
    case 32: return kernel_smem_bytes<0, 32>(m);
    case 108: return kernel_smem_bytes<1, 8>(m);
    case 116: return kernel_smem_bytes<1, 16>(m);
    case 132: return kernel_smem_bytes<1, 32>(m);
    case 208: return kernel_smem_bytes<2, 8>(m);
    case 216: return kernel_smem_bytes<2, 16>(m);
    case 232: return kernel_smem_bytes<2, 32>(m);
    case 308: return kernel_smem_bytes<3, 8>(m);
    case 316: return kernel_smem_bytes<3, 16>(m);
    default: return kernel_smem_bytes<3, 32>(m);
    }
}

cudaError_t launch_fit(int model, int lanes, const FitArgs &a, const GuessArgs &ga, int sms, cudaStream_t s,
                       LaunchInfo *info) {
    switch (model) {
    case kGaussian:
        return launch_model<kGaussian>(a, ga, lanes, sms, s, info);
    case kLorentzian:
        return launch_model<kLorentzian>(a, ga, lanes, sms, s, info);
    case kPseudoVoigt:
        return launch_model<kPseudoVoigt>(a, ga, lanes, sms, s, info);
    case kTwoLorentzian:
        return launch_model<kTwoLorentzian>(a, ga, lanes, sms, s, info);
    default:
        return cudaErrorInvalidValue;
    }
}

} // namespace bf
