// Device building blocks for the batchfit B200 kernels: thread-group views over
// warp lanes, exactly rounded float helpers, MUFU approximations, and the
// compensated reduce-scatter used by every LM pass.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bf {

// ------------------------------------------------------------ thread groups --
// A group of G (8, 16 or 32) consecutive lanes of one warp that cooperates on one
// fit.  Several groups of a warp proceed independently (each has its own mask).
template <int G> struct Group {
    static_assert(G == 8 || G == 16 || G == 32, "group size");
    static constexpr int size = G;
    unsigned lane;  // 0..G-1
    unsigned base;  // first warp lane of this group
    unsigned mask;  // member lanes within the warp
    __device__ __forceinline__ Group() {
        const unsigned wl = threadIdx.x & 31u;
        lane = wl & unsigned(G - 1);
        base = wl & ~unsigned(G - 1);
        mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << base);
    }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    template <class T> __device__ __forceinline__ T bcast(T v, int src) const {
        return __shfl_sync(mask, v, src, G);
    }
    template <class T> __device__ __forceinline__ T xor_(T v, int o) const {
        return __shfl_xor_sync(mask, v, o, G);
    }
    // Value of the previous / next group lane (a lane's own value at the ends).
    template <class T> __device__ __forceinline__ T prev(T v) const { return __shfl_up_sync(mask, v, 1, G); }
    template <class T> __device__ __forceinline__ T next(T v) const { return __shfl_down_sync(mask, v, 1, G); }
    // Bit i set <=> pred true on group lane i.
    __device__ __forceinline__ unsigned ballot(bool p) const {
        return (__ballot_sync(mask, p) & mask) >> base;
    }
    __device__ __forceinline__ bool any(bool p) const { return ballot(p) != 0u; }
    __device__ __forceinline__ bool all(bool p) const { return ballot(!p) == 0u; }
};

// A whole CTA of THREADS threads cooperating on one fit (the long-spectrum path):
// the same members the per-fit control code uses from a Group.
template <int THREADS> struct CtaGroup {
    static constexpr int size = THREADS;
    unsigned lane; // threadIdx.x
    __device__ __forceinline__ CtaGroup() : lane(threadIdx.x) {}
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// ----------------------------------------------------- exactly rounded ops --
// The data-only guess must round every operation as the reference's float C++
// does on the host (no contraction), so it uses the _rn intrinsics throughout.
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }
// a / 2 exactly as the division rounds it: a / 2 and a * 0.5 are the same real
// number, so their correctly rounded results are equal (subnormals included).
__device__ __forceinline__ float rhalf(float a) { return __fmul_rn(a, 0.5f); }

// std::midpoint for float (C++20 [numeric.ops.midpoint]).
__device__ __forceinline__ float midpoint_rn(float a, float b) {
    const float lo = 1.17549435e-38f * 2.0f, hi = 3.40282347e+38f / 2.0f;
    const float aa = fabsf(a), ab = fabsf(b);
    if (aa <= hi && ab <= hi)
        return rhalf(radd(a, b));
    if (aa < lo)
        return radd(a, rhalf(b));
    if (ab < lo)
        return radd(rhalf(a), b);
    return radd(rhalf(a), rhalf(b));
}

// std::lerp for float as libstdc++ evaluates it (C++20 [c.math.lerp]).
// Both formulas are evaluated and the result selected, so that the groups of a warp
// do not split on the branches.
__device__ __forceinline__ float lerp_rn(float a, float b, float t) {
    const bool straddle = (a <= 0.0f && b >= 0.0f) || (a >= 0.0f && b <= 0.0f);
    const float across = radd(rmul(t, b), rmul(rsub(1.0f, t), a));
    const float v = radd(a, rmul(t, rsub(b, a)));
    const float bounded = (t > 1.0f) == (b > a) ? (b < v ? v : b) : (b > v ? v : b);
    return straddle ? across : (t == 1.0f ? b : bounded);
}

// std::min / std::max argument semantics (ties keep the first argument).
__device__ __forceinline__ float smin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float sclamp(float v, float lo, float hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}
__device__ __forceinline__ double dclamp(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

// --------------------------------------------------------- MUFU helpers --
__device__ __forceinline__ float ex2_approx(float v) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}
__device__ __forceinline__ float rcp_approx(float v) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}

// ------------------------------------------------- packed float32 pairs --
// sm_100 f32x2 arithmetic: one instruction computes two IEEE float32 results, each
// rounded to nearest exactly as the scalar operation would be.  The LM pass
// evaluates two adjacent points per lane with these, halving its issue slots.
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(d)
        : "l"(*reinterpret_cast<const unsigned long long *>(&a)),
          "l"(*reinterpret_cast<const unsigned long long *>(&b)));
    return *reinterpret_cast<const float2 *>(&d);
}
__device__ __forceinline__ float2 ex2_approx2(float2 v) { return make_float2(ex2_approx(v.x), ex2_approx(v.y)); }
__device__ __forceinline__ float2 rcp_approx2(float2 v) { return make_float2(rcp_approx(v.x), rcp_approx(v.y)); }

// --------------------------------------------------- compensated sums --
// Knuth two-sum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

__host__ __device__ inline int round_up(int v, int a) { return (v + a - 1) / a * a; }
// Edge samples per side of the data-only guess: max(1, M/10) (initial_guess.hpp:142).
__host__ __device__ inline int edge_count(int m) { return m / 10 > 1 ? m / 10 : 1; }
__host__ __device__ inline int pow2_at_least(int v) {
    int p = 1;
    while (p < v)
        p <<= 1;
    return p;
}

__host__ __device__ constexpr int pow2ceil(int v) {
    int p = 1;
    while (p < v)
        p <<= 1;
    return p;
}

// Slots of a reduce-scatter of v sums over G lanes: a multiple of G when v >= G
// (every level halves a lane's slots), else a power of two dividing G (replicated
// owners).  Padding slots are zeros; the butterfly pairs the same lanes in the same
// order whatever the padding, so the reduced values do not depend on it.
__host__ __device__ constexpr int reduce_slots(int v, int g) { return v >= g ? (v + g - 1) / g * g : pow2ceil(v); }

// Reduce-scatter of KP per-lane partial sums over the G lanes of a group with a
// two-sum at every tree level.  At each level a lane keeps half of its live slots
// and ships the other half to its partner, so the shuffle count is ~KP instead of
// KP*log2(G).  Each reduced slot (hi + lo) is written once as a double to out[].
template <int G, int KP, int O, int S> struct ReduceLevel {
    __device__ __forceinline__ static void run(const Group<G> &g, float (&hi)[KP], float (&lo)[KP],
                                               int &slot_base, bool first) {
        if constexpr (O >= 1) {
            if constexpr (S > 1) {
                const bool up = (g.lane & unsigned(O)) != 0u;
#pragma unroll
                for (int i = 0; i < S / 2; ++i) {
                    const float send_h = up ? hi[i] : hi[i + S / 2];
                    const float keep_h = up ? hi[i + S / 2] : hi[i];
                    const float send_l = up ? lo[i] : lo[i + S / 2];
                    const float keep_l = up ? lo[i + S / 2] : lo[i];
                    const float recv_h = g.xor_(send_h, O);
                    const float recv_l = first ? 0.0f : g.xor_(send_l, O);
                    float s, e;
                    two_sum(keep_h, recv_h, s, e);
                    hi[i] = s;
                    lo[i] = __fadd_rn(__fadd_rn(keep_l, recv_l), e);
                }
                if (up)
                    slot_base += S / 2;
                ReduceLevel<G, KP, O / 2, S / 2>::run(g, hi, lo, slot_base, false);
            } else {
                const float recv_h = g.xor_(hi[0], O);
                const float recv_l = first ? 0.0f : g.xor_(lo[0], O);
                float s, e;
                two_sum(hi[0], recv_h, s, e);
                hi[0] = s;
                lo[0] = __fadd_rn(__fadd_rn(lo[0], recv_l), e);
                ReduceLevel<G, KP, O / 2, 1>::run(g, hi, lo, slot_base, false);
            }
        }
    }
};

// Number of slots each lane owns after the reduce-scatter, and the lane-bit mask
// below which owners are replicas (when KP < G).
template <int G, int KP> struct ReduceShape {
    static constexpr int owned = KP >= G ? KP / G : 1;
    static constexpr int replicas = KP >= G ? 1 : G / KP;
};

// hi[]/lo[] enter as each lane's compensated partial sums (value = hi + lo).
// Returns whether every reduced slot this lane owns is finite.
template <int G, int KP>
__device__ __forceinline__ bool reduce_scatter_store(const Group<G> &g, float (&hi)[KP], float (&lo)[KP],
                                                     double *out, int k_used) {
    int slot_base = 0;
    ReduceLevel<G, KP, G / 2, KP>::run(g, hi, lo, slot_base, false);
    constexpr int owned = ReduceShape<G, KP>::owned;
    constexpr int replicas = ReduceShape<G, KP>::replicas;
    bool finite = true;
#pragma unroll
    for (int i = 0; i < owned; ++i) {
        const double v = double(hi[i]) + double(lo[i]);
        if (slot_base + i < k_used) {
            finite = finite && isfinite(v);
            if ((g.lane & unsigned(replicas - 1)) == 0u)
                out[slot_base + i] = v;
        }
    }
    return finite;
}

} // namespace bf
