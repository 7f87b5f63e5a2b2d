// Fits in normalised coordinates from float64 data (include/batchfit_cuda.h,
// "Physical units").
//
// The reference prepares each spectrum in double before converting it to float
// (struct Coordinates, include/batchfit/coordinates.hpp:15-113): x is centred on the
// midpoint of its range and scaled by the half range, y by the spectrum's largest
// |y|; the fit runs in those units and parameters, chi-squared and covariance are
// mapped back to physical units in double.  Here both steps are kernels: one warp
// normalises one spectrum (float64 in, float32 out), the fit is the ordinary
// device-memory fit, and one thread per fit maps its results back.
#include "batchfit_cuda.h"
#include "bf_context.h"

#include <cmath>
#include <cstring>
#include <string>

namespace {

using bf::host::report;
using bf::host::report_cuda;

int parameters(int model) { return model == 2 ? 4 : model == 3 ? 8 : 3; }

struct XRange {
    double lo, hi;
    int finite;
};

// Range and finiteness of x (Coordinates::from, coordinates.hpp:17-30): one block.
__global__ void __launch_bounds__(256) x_range_kernel(const double *x, uint32_t m, XRange *out) {
    __shared__ double lo_s[8], hi_s[8];
    __shared__ int fin_s[8];
    double lo = x[0], hi = x[0];
    int fin = 1;
    for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) {
        const double v = x[j];
        fin &= isfinite(v) ? 1 : 0;
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    for (int o = 16; o >= 1; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        fin &= __shfl_xor_sync(0xffffffffu, fin, o);
    }
    const int w = threadIdx.x / 32;
    if ((threadIdx.x & 31) == 0) {
        lo_s[w] = lo;
        hi_s[w] = hi;
        fin_s[w] = fin;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < int(blockDim.x / 32); ++i) {
            lo = fmin(lo, lo_s[i]);
            hi = fmax(hi, hi_s[i]);
            fin &= fin_s[i];
        }
        *out = XRange{lo, hi, fin};
    }
}

struct Coords {
    double origin, x_scale;
};

// x in fitted units.
__global__ void normalize_x_kernel(const double *x, uint32_t m, Coords c, float *xn) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
        xn[j] = float((x[j] - c.origin) / c.x_scale);
}

// One warp per spectrum: y_scale = max|y| (1 when all zero), y / y_scale as float32,
// the initial values in fitted units (Coordinates::normalize, coordinates.hpp:63-86).
template <int P>
__global__ void __launch_bounds__(256) normalize_y_kernel(const double *y, uint64_t n, uint32_t m,
                                                          const double *p0, Coords c, float *yn, float *p0n,
                                                          double *y_scale, int *nonfinite) {
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const uint64_t warps = uint64_t(gridDim.x) * blockDim.x / 32;
    const unsigned lane = threadIdx.x & 31u;
    for (uint64_t f = warp; f < n; f += warps) {
        const double *row = y + f * m;
        double s = 0.0;
        int fin = 1;
        for (uint32_t j = lane; j < m; j += 32) {
            const double v = row[j];
            fin &= isfinite(v) ? 1 : 0;
            s = fmax(s, fabs(v));
        }
        for (int o = 16; o >= 1; o >>= 1) {
            s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
            fin &= __shfl_xor_sync(0xffffffffu, fin, o);
        }
        if (!fin && lane == 0)
            atomicOr(nonfinite, 1);
        const double scale = s > 0.0 ? s : 1.0;
        for (uint32_t j = lane; j < m; j += 32)
            yn[f * m + j] = float(row[j] / scale);
        if (lane == 0) {
            y_scale[f] = scale;
            if (p0) {
                const double *q = p0 + f * P;
                double r[P];
                for (int k = 0; k < P; ++k)
                    r[k] = q[k];
                r[0] /= scale;
                r[1] = (r[1] - c.origin) / c.x_scale;
                r[2] /= c.x_scale;
                if constexpr (P == 8) {
                    r[3] /= scale;
                    r[4] = (r[4] - c.origin) / c.x_scale;
                    r[5] /= c.x_scale;
                    r[6] = fma(q[7], c.origin, q[6]) / scale;
                    r[7] = q[7] * c.x_scale / scale;
                }
                for (int k = 0; k < P; ++k)
                    p0n[f * P + k] = float(r[k]);
            }
        }
    }
}

// One thread per fit: parameters, chi-squared and covariance in physical units
// (Coordinates::physical, physical_chi_squared, physical_covariance,
// coordinates.hpp:32-61,87-110); standard errors from the physical covariance.
template <int P>
__global__ void physical_kernel(uint64_t n, Coords c, const double *y_scale, const float *params,
                                const float *chi2, const float *cov, const int32_t *ustatus, double *params_out,
                                double *chi2_out, double *cov_out, double *se_out) {
    const uint64_t f = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (f >= n)
        return;
    const double ys = y_scale[f];
    double q[P], r[P];
    for (int k = 0; k < P; ++k)
        q[k] = params[f * P + k];
    for (int k = 0; k < P; ++k)
        r[k] = q[k];
    r[0] *= ys;
    r[1] = fma(r[1], c.x_scale, c.origin);
    r[2] *= c.x_scale;
    if constexpr (P == 8) {
        r[3] *= ys;
        r[4] = fma(r[4], c.x_scale, c.origin);
        r[5] *= c.x_scale;
        r[7] = q[7] * ys / c.x_scale;
        r[6] = fma(-r[7], c.origin, q[6] * ys);
    }
    for (int k = 0; k < P; ++k)
        params_out[f * P + k] = r[k];
    chi2_out[f] = (double(chi2[f]) * ys) * ys;
    if (!cov)
        return;
    // T: diagonal scales, plus the intercept/slope coupling of the linear baseline.
    double t[P][P] = {};
    for (int i = 0; i < P; ++i)
        t[i][i] = i == 0 ? ys : (i == 1 || i == 2) ? c.x_scale : 1.0;
    if constexpr (P == 8) {
        t[3][3] = ys;
        t[4][4] = t[5][5] = c.x_scale;
        t[6][6] = ys;
        t[6][7] = -c.origin * ys / c.x_scale;
        t[7][7] = ys / c.x_scale;
    }
    const float *cf = cov + f * P * P;
    for (int i = 0; i < P; ++i)
        for (int j = 0; j < P; ++j) {
            double s = 0.0;
            for (int k = 0; k < P; ++k)
                for (int l = 0; l < P; ++l)
                    s += t[i][k] * double(cf[k * P + l]) * t[j][l];
            cov_out[(f * P + i) * P + j] = s;
        }
    for (int i = 0; i < P; ++i)
        se_out[f * P + i] = ustatus[f] == 0 ? sqrt(cov_out[(f * P + i) * P + i]) : double(NAN);
}

template <int P> cudaError_t launch_normalize(const bf_physical_args &a, Coords c, float *yn, float *p0n,
                                               double *ys, int *flag, cudaStream_t st) {
    normalize_y_kernel<P><<<2048, 256, 0, st>>>(a.y, a.n, a.m, a.p0, c, yn, p0n, ys, flag);
    return cudaGetLastError();
}

template <int P> cudaError_t launch_physical(const bf_physical_args &a, Coords c, const double *ys,
                                              const bf_fit_outputs &o, const bf_physical_outputs &out,
                                              cudaStream_t st) {
    const unsigned blocks = unsigned((a.n + 127) / 128);
    physical_kernel<P><<<blocks, 128, 0, st>>>(a.n, c, ys, o.params, o.chi2, a.uncertainties ? o.covariance : nullptr,
                                               o.uncertainty_status, out.params, out.chi2,
                                               a.uncertainties ? out.covariance : nullptr, out.standard_errors);
    return cudaGetLastError();
}

struct Scratch {
    bf::host::DeviceBuffer buf;
};

} // namespace

extern "C" {

int bf_cuda_fit_physical(bf_cuda_context *ctx, const bf_physical_args *args, const bf_physical_outputs *out) {
    if (!ctx || !args || !out)
        return report(BF_ERR_INVALID_ARGUMENT, "null argument");
    const bf_physical_args &a = *args;
    if (a.model < 0 || a.model > 3)
        return report(BF_ERR_INVALID_ARGUMENT, "unknown model id");
    if (a.m == 0 || !a.x)
        return report(BF_ERR_INVALID_ARGUMENT, "normalization requires matching nonempty x/y");
    if (a.n == 0)
        return BF_OK;
    if (!a.y || !out->params || !out->status || !out->iterations || !out->chi2 ||
        (a.uncertainties && (!out->covariance || !out->standard_errors || !out->uncertainty_status)))
        return report(BF_ERR_INVALID_ARGUMENT, "inputs and outputs are required");
    const int p = parameters(a.model);
    const uint64_t n = a.n, m = a.m;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess)
        return report_cuda(e, "cudaSetDevice");
    // Scratch: x, y and p0 in fitted units, y scales, float outputs, flags.
    auto al = [](size_t v) { return (v + 255) / 256 * 256; };
    const size_t b_x = al(m * 4), b_y = al(n * m * 4), b_p0 = a.p0 ? al(n * p * 4) : 0, b_ys = al(n * 8),
                 b_par = al(n * p * 4), b_n4 = al(n * 4), b_cov = a.uncertainties ? al(n * p * p * 4) : 0,
                 b_se = a.uncertainties ? al(n * p * 4) : 0, b_flag = 256;
    const size_t total = b_x + b_y + b_p0 + b_ys + b_par + 3 * b_n4 + b_cov + b_se + b_flag;
    bf::host::DeviceBuffer scratch;
    e = scratch.reserve(total);
    if (e != cudaSuccess)
        return report_cuda(e, "normalisation scratch");
    char *at = static_cast<char *>(scratch.ptr);
    auto take = [&](size_t bytes) {
        char *here = at;
        at += bytes;
        return here;
    };
    float *xn = reinterpret_cast<float *>(take(b_x));
    float *yn = reinterpret_cast<float *>(take(b_y));
    float *p0n = a.p0 ? reinterpret_cast<float *>(take(b_p0)) : nullptr;
    double *ys = reinterpret_cast<double *>(take(b_ys));
    bf_fit_outputs o{};
    o.params = reinterpret_cast<float *>(take(b_par));
    o.chi2 = reinterpret_cast<float *>(take(b_n4));
    o.status = out->status;
    o.iterations = out->iterations;
    float *cov32 = a.uncertainties ? reinterpret_cast<float *>(take(b_cov)) : nullptr;
    float *se32 = a.uncertainties ? reinterpret_cast<float *>(take(b_se)) : nullptr;
    o.covariance = cov32;
    o.standard_errors = se32;
    o.uncertainty_status = out->uncertainty_status;
    take(2 * b_n4);
    char *flags = take(b_flag);
    XRange *xr = reinterpret_cast<XRange *>(flags);
    int *nonfinite = reinterpret_cast<int *>(flags + 64);
    cudaStream_t st = ctx->stream[0];
    XRange h{};
    e = cudaMemsetAsync(nonfinite, 0, sizeof(int), st);
    if (e == cudaSuccess) {
        x_range_kernel<<<1, 256, 0, st>>>(a.x, a.m, xr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&h, xr, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return report_cuda(e, "x range");
    const double half = h.hi / 2 - h.lo / 2;
    if (!h.finite)
        return report(BF_ERR_INVALID_ARGUMENT, "normalization requires finite inputs");
    if (!(half > 0) || !std::isfinite(half))
        return report(BF_ERR_INVALID_ARGUMENT, "normalization requires a resolved x range");
    // std::midpoint(lo, hi) for double (C++20 [numeric.ops.midpoint]).
    auto midpoint = [](double u, double v) {
        const double lo_lim = 2.2250738585072014e-308 * 2, hi_lim = 1.7976931348623157e308 / 2;
        if (std::fabs(u) <= hi_lim && std::fabs(v) <= hi_lim)
            return (u + v) / 2;
        if (std::fabs(u) < lo_lim)
            return u + v / 2;
        if (std::fabs(v) < lo_lim)
            return u / 2 + v;
        return u / 2 + v / 2;
    };
    const Coords c{midpoint(h.lo, h.hi), half};
    normalize_x_kernel<<<unsigned((m + 255) / 256), 256, 0, st>>>(a.x, a.m, c, xn);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = a.model == 2 ? launch_normalize<4>(a, c, yn, p0n, ys, nonfinite, st)
            : a.model == 3 ? launch_normalize<8>(a, c, yn, p0n, ys, nonfinite, st)
                           : launch_normalize<3>(a, c, yn, p0n, ys, nonfinite, st);
    int bad = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&bad, nonfinite, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return report_cuda(e, "normalisation");
    if (bad)
        return report(BF_ERR_INVALID_ARGUMENT, "normalization requires finite inputs");
    bf_fit_args fa{};
    fa.model = a.model;
    fa.n = n;
    fa.m = a.m;
    fa.x = xn;
    fa.y = yn;
    fa.p0 = p0n;
    fa.memory = BF_MEMORY_DEVICE;
    fa.uncertainties = a.uncertainties;
    fa.group_lanes = a.group_lanes;
    fa.options = a.options;
    int rc = bf_cuda_fit(ctx, &fa, &o);
    if (rc != BF_OK)
        return rc;
    e = a.model == 2 ? launch_physical<4>(a, c, ys, o, *out, st)
        : a.model == 3 ? launch_physical<8>(a, c, ys, o, *out, st)
                       : launch_physical<3>(a, c, ys, o, *out, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return report_cuda(e, "physical units");
    return BF_OK;
}

} // extern "C"
