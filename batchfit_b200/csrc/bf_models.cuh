// The four spectral models on the device: fused value + analytic Jacobian for the
// LM passes.  Formulas follow the reference's shared definitions
// (include/batchfit/models.hpp:78-185); the arithmetic is arranged for the GPU:
// one reciprocal of the width per pass, exp(-4 ln2 z^2) as ex2(-4 z^2) on the
// MUFU unit, and 1/(1+u) as a MUFU reciprocal.
//
// Each model also evaluates two points at once (residual2) with sm_100 packed
// float32 pairs: the same operations in the same order as residual, so each point
// of a pair rounds exactly as it would alone; only the MUFU approximations stay
// per value.
#pragma once

#include "bf_device.cuh"

namespace bf {

enum ModelId : int { kGaussian = 0, kLorentzian = 1, kPseudoVoigt = 2, kTwoLorentzian = 3 };

__host__ __device__ constexpr int model_parameters(int model) {
    return model == kPseudoVoigt ? 4 : model == kTwoLorentzian ? 8 : 3;
}

template <int MODEL> struct Model;

// amplitude * exp(-z^2/2), z = (x - center)/sigma   (models.hpp:88-99)
template <> struct Model<kGaussian> {
    static constexpr int P = 3;
    static constexpr bool paired = false;
    // FWHM/sigma for unresolved-peak detection (solver.hpp:86).
    static constexpr float width_factor = 2.354820045030949382f;
    struct Pre {
        float a, c, iw, aiw;
    };
    __device__ __forceinline__ static Pre prepare(const float *p) {
        const float iw = 1.0f / p[2];
        return {p[0], p[1], iw, p[0] * iw};
    }
    __device__ __forceinline__ static float residual(const Pre &q, float x, float y, float *J) {
        const float z = (x - q.c) * q.iw;
        // exp(-z^2/2) = 2^(-log2(e)/2 * z^2)
        const float g = ex2_approx(z * z * -0.72134752044448170368f);
        const float t = q.aiw * g * z;
        J[0] = g;
        J[1] = t;
        J[2] = t * z;
        return fmaf(-q.a, g, y);
    }
    struct Pre2 {
        float2 c, iw, aiw, na, k;
    };
    __device__ __forceinline__ static Pre2 prepare2(const float *p) {
        const Pre q = prepare(p);
        return {splat2(q.c), splat2(q.iw), splat2(q.aiw), splat2(-q.a), splat2(-0.72134752044448170368f)};
    }
    __device__ __forceinline__ static float2 residual2(const Pre2 &q, float2 x, float2 y, float2 *J) {
        const float2 z = mul2(sub2(x, q.c), q.iw);
        const float2 g = ex2_approx2(mul2(mul2(z, z), q.k));
        const float2 t = mul2(mul2(q.aiw, g), z);
        J[0] = g;
        J[1] = t;
        J[2] = mul2(t, z);
        return fma2(q.na, g, y);
    }
};

// amplitude / (1 + z^2), z = (x - center)/hwhm   (models.hpp:112-124)
template <> struct Model<kLorentzian> {
    static constexpr int P = 3;
    static constexpr bool paired = false;
    static constexpr float width_factor = 2.0f;
    struct Pre {
        float a, c, iw, a2iw;
    };
    __device__ __forceinline__ static Pre prepare(const float *p) {
        const float iw = 1.0f / p[2];
        return {p[0], p[1], iw, 2.0f * p[0] * iw};
    }
    __device__ __forceinline__ static float residual(const Pre &q, float x, float y, float *J) {
        const float z = (x - q.c) * q.iw;
        const float s = rcp_approx(fmaf(z, z, 1.0f));
        const float t = q.a2iw * s * s * z;
        J[0] = s;
        J[1] = t;
        J[2] = t * z;
        return fmaf(-q.a, s, y);
    }
    struct Pre2 {
        float2 c, iw, a2iw, na, one;
    };
    __device__ __forceinline__ static Pre2 prepare2(const float *p) {
        const Pre q = prepare(p);
        return {splat2(q.c), splat2(q.iw), splat2(q.a2iw), splat2(-q.a), splat2(1.0f)};
    }
    __device__ __forceinline__ static float2 residual2(const Pre2 &q, float2 x, float2 y, float2 *J) {
        const float2 z = mul2(sub2(x, q.c), q.iw);
        const float2 s = rcp_approx2(fma2(z, z, q.one));
        const float2 t = mul2(mul2(mul2(q.a2iw, s), s), z);
        J[0] = s;
        J[1] = t;
        J[2] = mul2(t, z);
        return fma2(q.na, s, y);
    }
};

// amplitude * ((1-eta) exp(-4 ln2 z^2) + eta / (1 + 4 z^2)), z = (x - center)/fwhm
// (models.hpp:138-156)
template <> struct Model<kPseudoVoigt> {
    static constexpr int P = 4;
    static constexpr bool paired = false;
    static constexpr float width_factor = 1.0f;
    struct Pre {
        float a, c, iw, eta, kl, kg; // kl = 8 a eta / w, kg = 8 a (1-eta) ln2 / w
    };
    __device__ __forceinline__ static Pre prepare(const float *p) {
        const float iw = 1.0f / p[2];
        const float a8iw = 8.0f * p[0] * iw;
        return {p[0], p[1], iw, p[3], a8iw * p[3], a8iw * ((1.0f - p[3]) * 0.69314718055994530942f)};
    }
    __device__ __forceinline__ static float residual(const Pre &q, float x, float y, float *J) {
        const float z = (x - q.c) * q.iw;
        const float z2 = z * z;
        const float g = ex2_approx(-4.0f * z2); // exp(-4 ln2 z^2) == 2^(-4 z^2)
        const float l = rcp_approx(fmaf(4.0f, z2, 1.0f));
        const float d = l - g;
        const float s = fmaf(q.eta, d, g); // (1-eta) g + eta l
        // df/dc = 8a/w z ((1-eta) ln2 g + eta l^2)
        const float t = fmaf(q.kl * l, l, q.kg * g) * z;
        J[0] = s;
        J[1] = t;
        J[2] = t * z;
        J[3] = q.a * d;
        return fmaf(-q.a, s, y);
    }
    struct Pre2 {
        float2 c, iw, eta, kl, kg, a, na, m4, p4, one;
    };
    __device__ __forceinline__ static Pre2 prepare2(const float *p) {
        const Pre q = prepare(p);
        return {splat2(q.c),  splat2(q.iw), splat2(q.eta),  splat2(q.kl),  splat2(q.kg),
                splat2(q.a),  splat2(-q.a), splat2(-4.0f), splat2(4.0f), splat2(1.0f)};
    }
    __device__ __forceinline__ static float2 residual2(const Pre2 &q, float2 x, float2 y, float2 *J) {
        const float2 z = mul2(sub2(x, q.c), q.iw);
        const float2 z2 = mul2(z, z);
        const float2 g = ex2_approx2(mul2(q.m4, z2));
        const float2 l = rcp_approx2(fma2(q.p4, z2, q.one));
        const float2 d = sub2(l, g);
        const float2 s = fma2(q.eta, d, g);
        const float2 t = mul2(fma2(mul2(q.kl, l), l, mul2(q.kg, g)), z);
        J[0] = s;
        J[1] = t;
        J[2] = mul2(t, z);
        J[3] = mul2(q.a, d);
        return fma2(q.na, s, y);
    }
};

// Two Lorentzians plus intercept + slope * x   (models.hpp:174-184)
template <> struct Model<kTwoLorentzian> {
    static constexpr int P = 8;
    static constexpr bool paired = true;
    static constexpr float width_factor = 2.0f;
    struct Pre {
        float a1, c1, iw1, k1, a2, c2, iw2, k2, b0, b1;
    };
    __device__ __forceinline__ static Pre prepare(const float *p) {
        const float iw1 = 1.0f / p[2], iw2 = 1.0f / p[5];
        return {p[0], p[1], iw1, 2.0f * p[0] * iw1, p[3], p[4], iw2, 2.0f * p[3] * iw2, p[6], p[7]};
    }
    __device__ __forceinline__ static float residual(const Pre &q, float x, float y, float *J) {
        const float z1 = (x - q.c1) * q.iw1;
        const float s1 = rcp_approx(fmaf(z1, z1, 1.0f));
        const float t1 = q.k1 * s1 * s1 * z1;
        const float z2 = (x - q.c2) * q.iw2;
        const float s2 = rcp_approx(fmaf(z2, z2, 1.0f));
        const float t2 = q.k2 * s2 * s2 * z2;
        J[0] = s1;
        J[1] = t1;
        J[2] = t1 * z1;
        J[3] = s2;
        J[4] = t2;
        J[5] = t2 * z2;
        J[6] = 1.0f;
        J[7] = x;
        return y - fmaf(q.a1, s1, fmaf(q.a2, s2, fmaf(q.b1, x, q.b0)));
    }
    struct Pre2 {
        float2 a1, c1, iw1, k1, a2, c2, iw2, k2, b0, b1, one;
    };
    __device__ __forceinline__ static Pre2 prepare2(const float *p) {
        const Pre q = prepare(p);
        return {splat2(q.a1), splat2(q.c1), splat2(q.iw1), splat2(q.k1), splat2(q.a2), splat2(q.c2),
                splat2(q.iw2), splat2(q.k2), splat2(q.b0), splat2(q.b1), splat2(1.0f)};
    }
    __device__ __forceinline__ static float2 residual2(const Pre2 &q, float2 x, float2 y, float2 *J) {
        const float2 z1 = mul2(sub2(x, q.c1), q.iw1);
        const float2 s1 = rcp_approx2(fma2(z1, z1, q.one));
        const float2 t1 = mul2(mul2(mul2(q.k1, s1), s1), z1);
        const float2 z2 = mul2(sub2(x, q.c2), q.iw2);
        const float2 s2 = rcp_approx2(fma2(z2, z2, q.one));
        const float2 t2 = mul2(mul2(mul2(q.k2, s2), s2), z2);
        J[0] = s1;
        J[1] = t1;
        J[2] = mul2(t1, z1);
        J[3] = s2;
        J[4] = t2;
        J[5] = mul2(t2, z2);
        J[6] = q.one;
        J[7] = x;
        return sub2(y, fma2(q.a1, s1, fma2(q.a2, s2, fma2(q.b1, x, q.b0))));
    }
};

} // namespace bf
