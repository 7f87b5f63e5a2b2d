// Data-only initial guess on the device, one thread group per spectrum.
//
// Restates initial_guess<float,Model> (include/batchfit/cpu/initial_guess.hpp:120-249)
// with group-parallel searches, and rounds every operation exactly as the
// reference's float C++ does (the _rn intrinsics: no contraction).  Its outputs
// and status equal the reference's float guess bit for bit; the parallel searches
// keep the reference's tie rules (first maximum / first minimum in index order).
#pragma once

#include <type_traits>

#include "bf_device.cuh"
#include "bf_models.cuh"

namespace bf {

enum GuessStatus : int { kGuessSuccess = 0, kGuessInvalid = 1, kGuessNoPeak = 2, kGuessInsufficient = 3 };

// Ascending bitonic sort of `batches` consecutive arrays of n (power of two) floats.
// Index arithmetic is shifts and masks only (n is a power of two).
template <int G>
__device__ __forceinline__ void bitonic_sort(const Group<G> &g, float *buf, int n, int batches) {
    const int half_shift = 31 - __clz(n > 1 ? n >> 1 : 1);
    const int half_mask = (n >> 1) - 1;
    const int pairs = (n >> 1) * batches;
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = int(g.lane); t < pairs; t += G) {
                const int b = t >> half_shift, u = t & half_mask;
                const int i = ((u & ~(j - 1)) << 1) | (u & (j - 1));
                float *a = buf + (b << (half_shift + 1));
                const float lo = a[i], hi = a[i | j];
                const bool ascending = (i & k) == 0;
                if (ascending ? (lo > hi) : (lo < hi)) {
                    a[i] = hi;
                    a[i | j] = lo;
                }
            }
            g.sync();
        }
    }
}

// Sort a bitonic sequence of n (power of two) floats ascending.
template <int G> __device__ __forceinline__ void bitonic_merge(const Group<G> &g, float *buf, int n) {
    for (int j = n >> 1; j > 0; j >>= 1) {
        for (int t = int(g.lane); t < (n >> 1); t += G) {
            const int i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
            const float lo = buf[i], hi = buf[i | j];
            if (lo > hi) {
                buf[i] = hi;
                buf[i | j] = lo;
            }
        }
        g.sync();
    }
}

// ------------------------------------------------- sorting in registers --
// N = G*V values in a blocked layout: group lane l holds elements [l*V, l*V+V).
// Compare-exchanges across lanes use shuffles, within a lane plain min/max; the
// network is fully unrolled (k, j are compile-time after unrolling).
__device__ __forceinline__ void cmpx(float &lo, float &hi, bool ascending) {
    const float a = lo, b = hi;
    lo = ascending ? fminf(a, b) : fmaxf(a, b);
    hi = ascending ? fmaxf(a, b) : fminf(a, b);
}

template <int G, int V>
__device__ __forceinline__ void reg_stage(const Group<G> &g, float (&v)[V], int k, int j, bool merge_only) {
    if (j >= V) {
        const int lx = j / V;
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const int e = int(g.lane) * V + i;
            const bool ascending = merge_only || (e & k) == 0;
            const bool keep_min = ascending == ((e & j) == 0);
            const float o = g.xor_(v[i], lx);
            v[i] = keep_min ? fminf(v[i], o) : fmaxf(v[i], o);
        }
    } else {
#pragma unroll
        for (int i = 0; i < V; ++i) {
            if ((i & j) == 0) {
                const int e = int(g.lane) * V + i;
                cmpx(v[i], v[i | j], merge_only || (e & k) == 0);
            }
        }
    }
}

// Ascending bitonic sort of G*V values.
template <int G, int V> __device__ __forceinline__ void reg_sort(const Group<G> &g, float (&v)[V]) {
    constexpr int N = G * V;
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
            reg_stage<G, V>(g, v, k, j, false);
}

// Ascending sort of a bitonic sequence of G*V values (log2 N stages).
template <int G, int V> __device__ __forceinline__ void reg_merge(const Group<G> &g, float (&v)[V]) {
    constexpr int N = G * V;
#pragma unroll
    for (int j = N >> 1; j > 0; j >>= 1)
        reg_stage<G, V>(g, v, N, j, true);
}

// Store a blocked run (lane l holds elements l*V .. l*V+V-1) to a 16-byte aligned
// buffer, 16 bytes at a time when V allows.
template <int G, int V> __device__ __forceinline__ void store_run(const Group<G> &g, const float (&v)[V], float *out) {
    if constexpr (V % 4 == 0) {
        float4 *o = reinterpret_cast<float4 *>(out + int(g.lane) * V);
#pragma unroll
        for (int i = 0; i < V; i += 4)
            o[i / 4] = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    } else {
#pragma unroll
        for (int i = 0; i < V; ++i)
            out[int(g.lane) * V + i] = v[i];
    }
}

// Median of the union of sorted a[0..n) and b[0..n) (2n values, an even count):
// the midpoint of its n-1-th and n-th smallest.  One merge-path search splits off
// the n smallest (i from a, n-i from b); the n-1-th is the larger of the last ones
// taken, the n-th the smaller of the next ones.
__device__ __forceinline__ float union_median(const float *a, const float *b, int n) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int i = (lo + hi) >> 1;
        if (a[i] < b[n - 1 - i])
            lo = i + 1;
        else
            hi = i;
    }
    const float inf = __int_as_float(0x7f800000);
    const int j = n - lo;
    const float last = fmaxf(lo > 0 ? a[lo - 1] : -inf, j > 0 ? b[j - 1] : -inf);
    const float next = fminf(lo < n ? a[lo] : inf, j < n ? b[j] : inf);
    return midpoint_rn(last, next);
}

// detail::median on sorted values (initial_guess.hpp:25-30).
__device__ __forceinline__ float sorted_median(const float *a, int n) {
    return (n & 1) ? a[n / 2] : midpoint_rn(a[n / 2 - 1], a[n / 2]);
}

// signal[j] = y[j] - (level + slope*(x[j]-left_x))   (initial_guess.hpp:158-162).
// PRE: ys already holds the signal (the guess kernel overwrites its staged copy of
// the row once, with exactly these roundings), so a sample is one load.
template <int MODEL, bool PRE = false> struct Signal {
    const float *xs, *ys;
    float level, slope, left_x;
    int m;
    __device__ __forceinline__ float at(int j) const {
        if constexpr (PRE)
            return ys[j];
        else
            return raw_at(j);
    }
    __device__ __forceinline__ float raw_at(int j) const { return raw(ys[j], xs[j]); }
    // The signal of sample value yj at abscissa xj.
    __device__ __forceinline__ float raw(float yj, float xj) const {
        if constexpr (Model<MODEL>::paired)
            return rsub(yj, radd(level, rmul(slope, rsub(xj, left_x))));
        else
            return rsub(yj, level); // slope == 0: equal value (up to the sign of zero)
    }
    // detail::smooth (initial_guess.hpp:32-36).
    __device__ __forceinline__ float smooth(int j) const {
        if (j == 0 || j + 1 == m)
            return at(j);
        return smooth_interior(j);
    }
    __device__ __forceinline__ float smooth_interior(int j) const {
        return radd(radd(rmul(0.25f, at(j - 1)), rmul(0.5f, at(j))), rmul(0.25f, at(j + 1)));
    }
    // detail::raw_maximum (initial_guess.hpp:111-115): first max of s[j-1..j+1].
    __device__ __forceinline__ int raw_maximum(int j) const {
        int best = j - 1;
        float bv = at(j - 1);
        const float v0 = at(j), v1 = at(j + 1);
        if (bv < v0) {
            best = j;
            bv = v0;
        }
        if (bv < v1)
            best = j + 1;
        return best;
    }
};

// ------------------------------------------------------- chunked sweep --
// The tallest-smoothed-maximum sweep in 4-sample chunks.  Chunk c (samples 4c..4c+3)
// goes to group lane c mod G at step c / G; that lane also reads chunk c-1 and
// tests samples 4c-2..4c+1, whose smoothed values and smoothed neighbours need
// samples 4c-4..4c+3 only: no shuffles, and from a staged row (16-byte aligned,
// round_up(m, 4) floats) two 16-byte reads a step.  Chunks 0..m/4 cover every
// interior sample.
__host__ __device__ inline int chunk_steps(int m, int lanes) { return (m / 4 + lanes) / lanes; }
// Candidate-bit words per lane: 4 bits a step.
__host__ __device__ inline int chunk_words(int m, int lanes) { return (chunk_steps(m, lanes) + 7) / 8; }
// Sample tested as bit b of a lane's candidate bits.
__device__ __forceinline__ int chunk_sample(int lane, int b, int lanes) {
    return 4 * (lane + (b >> 2) * lanes) - 2 + (b & 3);
}

// One step of the chunked sweep for chunk c: cv[t] is the smoothed value of sample
// j = 4c-2+t when j is an interior smoothed local maximum (v > left, v >= right;
// initial_guess.hpp:173-174), else 0 (a value that never beats a height >= 0).
// `fin` accumulates whether the chunk's own samples are finite.  EDGE: the step
// may touch sample 0, sample m-1 or samples past the row (masked, unsmoothed ends).
// VEC: the row is staged (16-byte aligned, padded to round_up(m, 4)) and read 16
// bytes at a time, as y (SUB: the signal is y - level) or as the signal itself;
// otherwise the samples come one by one from the Signal `sig` (any alignment, no
// padding: samples outside the row are not read).
template <bool EDGE, bool SUB, bool VEC, class S>
__device__ __forceinline__ void chunk_step(const float4 *row, const S &sig, int m, float level, int c,
                                           float (&cv)[4], bool &fin) {
    const int j0 = 4 * c - 4;
    float s[8]; // samples 4c-4+i
    if constexpr (VEC) {
        const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float4 a = !EDGE || (c >= 1 && j0 < m) ? row[c - 1] : zero;
        const float4 b = !EDGE || j0 + 4 < m ? row[c] : zero;
        s[0] = a.x, s[1] = a.y, s[2] = a.z, s[3] = a.w, s[4] = b.x, s[5] = b.y, s[6] = b.z, s[7] = b.w;
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i)
            s[i] = !EDGE || (j0 + i >= 0 && j0 + i < m) ? sig.at(j0 + i) : 0.0f;
    }
    if constexpr (VEC && SUB) {
        // The signal of a baseline-only model, y - level (Signal::raw), two at a time.
#pragma unroll
        for (int i = 0; i < 8; i += 2) {
            const float2 d = sub2(make_float2(s[i], s[i + 1]), splat2(level));
            s[i] = d.x;
            s[i + 1] = d.y;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (EDGE && j0 + i >= m)
            s[i] = 0.0f; // the padding of the last chunk is not data
        if (i >= 4)
            fin = fin && fabsf(s[i]) <= 3.40282347e+38f;
    }
    // 0.25*s and 0.5*s of every sample, two samples per instruction.
    float q[8], h[8];
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        const float2 p = make_float2(s[i], s[i + 1]);
        const float2 pq = mul2(splat2(0.25f), p), ph = mul2(splat2(0.5f), p);
        q[i] = pq.x;
        q[i + 1] = pq.y;
        h[i] = ph.x;
        h[i + 1] = ph.y;
    }
    float v[6]; // smoothed samples 4c-3..4c+2, summed in detail::smooth's order
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        v[t] = radd(radd(q[t], h[t + 1]), q[t + 2]);
        if (EDGE && (j0 + 1 + t == 0 || j0 + 1 + t == m - 1))
            v[t] = s[t + 1];
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        bool peak = v[t + 1] > v[t] && v[t + 1] >= v[t + 2];
        if (EDGE)
            peak = peak && j0 + 2 + t >= 1 && j0 + 2 + t <= m - 2;
        cv[t] = peak ? v[t + 1] : 0.0f;
    }
}

// Tallest smoothed local maximum of the group lane's chunks (value and first
// index; index m when no positive one) and, with BITS, the lane's candidate bits
// (positive smoothed local maxima, bit 4k+t for sample 4(lane+kG)-2+t, words at
// bits[w*G]).  SUB: the row holds y and the signal is y - level.  Returns whether
// the lane's signal samples are finite.
template <int G, bool BITS, bool SUB, bool VEC, class S>
__device__ __forceinline__ bool chunk_sweep(const Group<G> &g, const S &sig, const float *signal, int m, float level,
                                            float &height, int &first, unsigned *bits) {
    const float4 *row = reinterpret_cast<const float4 *>(signal);
    const int steps = chunk_steps(m, G);
    bool fin = true;
    height = 0.0f;
    int best = -1;
    unsigned word = 0;
    auto visit = [&](auto edge, int k) {
        float cv[4];
        chunk_step<decltype(edge)::value, SUB, VEC>(row, sig, m, level, int(g.lane) + k * G, cv, fin);
        const float top = fmaxf(fmaxf(cv[0], cv[1]), fmaxf(cv[2], cv[3]));
        if (top > height) {
            height = top;
            best = k;
        }
        if constexpr (BITS) {
            word |= (unsigned(cv[0] > 0.0f) | unsigned(cv[1] > 0.0f) << 1 | unsigned(cv[2] > 0.0f) << 2 |
                     unsigned(cv[3] > 0.0f) << 3)
                    << (4 * (k & 7));
            if ((k & 7) == 7 || k + 1 == steps) {
                bits[(k >> 3) * G + int(g.lane)] = word;
                word = 0;
            }
        }
    };
    // Steps 1 <= k < inner touch neither end of the row for any lane (4G(k+1) < m):
    // those run branch-free, two per loop turn; the first and the last take the
    // masked step.
    const int inner = min(steps, (m - 1) / (4 * G));
    visit(std::true_type{}, 0);
#pragma unroll 2
    for (int k = 1; k < inner; ++k)
        visit(std::false_type{}, k);
    for (int k = inner > 1 ? inner : 1; k < steps; ++k)
        visit(std::true_type{}, k);
    first = m;
    if (best >= 0) {
        // The first sample of the best step that reaches the height.
        const int c = int(g.lane) + best * G;
        float cv[4];
        bool unused = true;
        chunk_step<true, SUB, VEC>(row, sig, m, level, c, cv, unused);
#pragma unroll
        for (int t = 3; t >= 0; --t)
            if (cv[t] == height)
                first = 4 * c - 2 + t;
    }
    return fin;
}

// Group argmax of (value, index): larger value wins, ties go to the smaller index.
template <int G> __device__ __forceinline__ void argmax_pair(const Group<G> &g, float &v, int &i) {
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) {
        const float ov = g.xor_(v, o);
        const int oi = g.xor_(i, o);
        if (ov > v || (ov == v && oi < i)) {
            v = ov;
            i = oi;
        }
    }
}

struct PeakFeature {
    float amplitude, center, width, left_radius, right_radius;
    bool valid;
};

// detail::peak (initial_guess.hpp:61-109) with the half-height walks done as
// group-parallel searches for the nearest sample at or below half height.
template <int G, class S>
__device__ PeakFeature find_peak(const Group<G> &g, const S &s, const float *xs, int index,
                                 int begin, int end, bool mirror) {
    PeakFeature r{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, false};
    r.amplitude = s.at(index);
    if (!(r.amplitude > 0.0f))
        return r;
    const float half = rhalf(r.amplitude);
    // while (left > begin && signal[left] > half) --left;
    int left = begin;
    for (int top = index - 1; top >= begin; top -= G) {
        const int pos = top - int(g.lane);
        const bool hit = pos >= begin && s.at(pos) <= half;
        const unsigned b = g.ballot(hit);
        if (b) {
            left = top - (__ffs(b) - 1);
            break;
        }
    }
    if (index == begin)
        left = index;
    // while (right < end && signal[right] > half) ++right;
    int right = end;
    for (int bot = index + 1; bot <= end; bot += G) {
        const int pos = bot + int(g.lane);
        const bool hit = pos <= end && s.at(pos) <= half;
        const unsigned b = g.ballot(hit);
        if (b) {
            right = bot + (__ffs(b) - 1);
            break;
        }
    }
    if (index == end)
        right = index;
    const bool has_left = s.at(left) <= half, has_right = s.at(right) <= half;
    if ((!has_left && (!mirror || begin == 0)) || (!has_right && (!mirror || end + 1 == s.m)) ||
        (!has_left && !has_right))
        return r;
    int low = index > 2 ? index - 2 : 0;
    int high = index + 2 < end ? index + 2 : end;
    const int low_limit = has_left ? left + 1 : begin;
    const int high_limit = has_right ? right - 1 : end;
    low = low < low_limit ? low_limit : low;
    high = high_limit < high ? high_limit : high;
    // Weighted centre over j = low..high (a window of at most 5 samples around the
    // index), detail::peak's loop: total += w; centre = lerp(centre, x[j], w/total)
    // for every w = max(0, s[j]) / amplitude > 0.  The divisions run side by side:
    // lane d takes sample index-2+d, every lane forms the running totals in the
    // window's order, and lane d divides its weight by its own running total.  Only
    // the lerp chain stays sequential.  Operations and order are the loop's.
    const int lane = int(g.lane);
    const int jl = index - 2 + lane;
    const bool mine = lane < 5 && jl >= low && jl <= high;
    const float w_own = mine ? rdiv(smax(0.0f, s.at(mine ? jl : index)), r.amplitude) : 0.0f;
    float w[5];
#pragma unroll
    for (int d = 0; d < 5; ++d)
        w[d] = g.bcast(w_own, d);
    float total = 0.0f, own_total = 1.0f;
#pragma unroll
    for (int d = 0; d < 5; ++d) {
        if (w[d] > 0.0f)
            total = radd(total, w[d]);
        if (d == lane)
            own_total = total;
    }
    const float q_own = w_own > 0.0f ? rdiv(w_own, own_total) : 0.0f;
    r.center = xs[index];
#pragma unroll
    for (int d = 0; d < 5; ++d) {
        const float q = g.bcast(q_own, d);
        const float xd = xs[w[d] > 0.0f ? index - 2 + d : index]; // in the window when taken
        if (w[d] > 0.0f)
            r.center = lerp_rn(r.center, xd, q);
    }
    // Both half-height crossings at once: lane 0 the left one, lane 1 the right one.
    float cross = __int_as_float(0x7fffffff);
    if ((lane == 0 && has_left) || (lane == 1 && has_right)) {
        const int a = lane == 0 ? left : right - 1, b = a + 1;
        const float den = rsub(s.at(b), s.at(a));
        if (isfinite(den) && den != 0.0f)
            cross = lerp_rn(xs[a], xs[b], rdiv(rsub(half, s.at(a)), den));
    }
    const float cross_left = g.bcast(cross, 0), cross_right = g.bcast(cross, 1);
    if (has_left)
        r.left_radius = rsub(r.center, cross_left);
    if (has_right)
        r.right_radius = rsub(cross_right, r.center);
    if (!has_left)
        r.left_radius = r.right_radius;
    if (!has_right)
        r.right_radius = r.left_radius;
    r.width = radd(r.left_radius, r.right_radius);
    r.valid = isfinite(r.center) && isfinite(r.width) && r.left_radius > 0.0f && r.right_radius > 0.0f;
    return r;
}

// Extrema of the smoothed signal over blocks of 32 samples (the last block may be
// short), for the prominence walks below, and the blocks' prefix and suffix minima
// (bmin, bmax, pmin, smin: four arrays of ceil(M/32) floats, back to back).  Lane l
// takes blocks l, l+G, ...
constexpr int kWalkBlock = 32;
__host__ __device__ inline int walk_blocks(int m) { return (m + kWalkBlock - 1) / kWalkBlock; }
// Scratch words of the second-peak search: four block arrays, then the chunked
// sweep's candidate bits (4 per step and lane; lane-wise words, word-major).
__host__ __device__ inline int second_peak_words(int m, int lanes) {
    return 4 * walk_blocks(m) + lanes * chunk_words(m, lanes);
}
template <int G, class S>
__device__ void block_extrema(const Group<G> &g, const S &s, float *bmin, float *bmax) {
    const int blocks = (s.m + kWalkBlock - 1) / kWalkBlock;
    for (int b = int(g.lane); b < blocks; b += G) {
        const int first = b * kWalkBlock, end = min(s.m, first + kWalkBlock);
        float lo = s.smooth(first), hi = lo;
        for (int j = first + 1; j < end; ++j) {
            const float v = s.smooth(j);
            lo = fminf(lo, v);
            hi = fmaxf(hi, v);
        }
        bmin[b] = lo;
        bmax[b] = hi;
    }
    g.sync();
    // Minima of the blocks up to b (prefix) and from b on (suffix).
    if (g.lane == 0) {
        float *pmin = bmax + blocks, *smin = pmin + blocks;
        float r = bmin[0];
        for (int b = 0; b < blocks; ++b) {
            r = fminf(r, bmin[b]);
            pmin[b] = r;
        }
        r = bmin[blocks - 1];
        for (int b = blocks - 1; b >= 0; --b) {
            r = fminf(r, bmin[b]);
            smin[b] = r;
        }
    }
    g.sync();
}

// A side of candidate `index` can clear the threshold only if the lowest sample
// anywhere on that side does (walk minima are at least the side minima, and the
// block prefix / suffix minima bound those from below): a necessary condition.
__device__ __forceinline__ bool may_be_prominent(const float *pmin, const float *smin, int m, int index,
                                                 float height, float threshold) {
    if (index < 1 || index + 1 >= m)
        return false;
    return rsub(height, pmin[(index - 1) / kWalkBlock]) > threshold &&
           rsub(height, smin[(index + 1) / kWalkBlock]) > threshold;
}

// detail::prominence(signal, index) > threshold (initial_guess.hpp:38-54), by one
// lane.  The reference walks outwards on each side while the smoothed signal stays
// at or below the start height, takes the side minima and returns height minus the
// larger minimum.  Rounding is monotone, so that exceeds the threshold iff on both
// sides some sample of the walk has height - sample > threshold.  Each walk stops
// at its first such sample (side passes) or at the reference's stop (side fails),
// and crosses whole blocks whose maximum is at most the height by their minimum.
template <class S>
__device__ bool prominent(const S &s, const float *bmin, const float *bmax, int index,
                          float threshold) {
    const float height = s.smooth(index);
    bool left = false;
    for (int j = index - 1; j >= 0;) {
        if ((j & (kWalkBlock - 1)) == kWalkBlock - 1 && bmax[j / kWalkBlock] <= height) {
            if (rsub(height, bmin[j / kWalkBlock]) > threshold) {
                left = true;
                break;
            }
            j -= kWalkBlock;
            continue;
        }
        const float v = s.smooth(j);
        if (v > height)
            break;
        if (rsub(height, v) > threshold) {
            left = true;
            break;
        }
        --j;
    }
    if (!left)
        return false;
    for (int j = index + 1; j < s.m;) {
        if ((j & (kWalkBlock - 1)) == 0 && bmax[j / kWalkBlock] <= height) {
            if (rsub(height, bmin[j / kWalkBlock]) > threshold)
                return true;
            j += kWalkBlock;
            continue;
        }
        const float v = s.smooth(j);
        if (v > height)
            return false;
        if (rsub(height, v) > threshold)
            return true;
        ++j;
    }
    return false;
}

// initial_guess<float,Model> for the spectrum ys[0..m).  `scratch` holds 2*n1 floats.
// Returns the GuessStatus; out[] receives the guessed parameters (NaN when the
// reference leaves them unset).
// V > 0: edge medians sorted in registers, G*V >= max(1, M/10) values per side;
// V == 0: the general shared-memory path (any M).  `scratch` holds
// 2*max(n1, G*V) floats.
template <int MODEL, int G, int V, bool PRE = false>
__device__ int initial_guess(const Group<G> &g, const XConst &xc, const float *xs, const float *ys,
                             bool y_finite, float *scratch, float *out) {
    constexpr int P = Model<MODEL>::P;
    constexpr bool paired = Model<MODEL>::paired;
    const float qnan = __int_as_float(0x7fffffff);
#pragma unroll
    for (int k = 0; k < P; ++k)
        out[k] = qnan;
    if (!xc.guess_ok || !y_finite)
        return kGuessInvalid;
    const int m = xc.m, count = xc.count, n1 = xc.n1;
    float left_level, right_level, baseline, slope, level, noise_median;
    if constexpr (V > 0) {
        // Edge medians (initial_guess.hpp:142-150): both sides sorted in registers;
        // the union median by a merge-path search over the two sorted runs.
        constexpr int N = G * V;
        float lv[V], rv[V];
        // Any placement sorts: lane l reads samples l, l+G, ... (consecutive lanes,
        // consecutive banks); the sorted values come out blocked, V per lane.
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const int e = i * G + int(g.lane);
            lv[i] = e < count ? ys[e] : __int_as_float(0x7f800000);
            rv[i] = e < count ? ys[m - count + e] : __int_as_float(0x7f800000);
        }
        reg_sort<G, V>(g, lv);
        reg_sort<G, V>(g, rv);
        store_run<G, V>(g, lv, scratch);
        store_run<G, V>(g, rv, scratch + N);
        g.sync();
        left_level = sorted_median(scratch, count);
        right_level = sorted_median(scratch + N, count);
        baseline = union_median(scratch, scratch + N, count);
        slope = paired ? rdiv(rsub(right_level, left_level), rsub(xc.right_x, xc.left_x)) : 0.0f;
        level = paired ? left_level : baseline;
        g.sync();
        // Absolute deviations of a sorted run from its median fall then rise: a
        // bitonic sequence, so a bitonic merge sorts each side.
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const int e = int(g.lane) * V + i;
            lv[i] = e < count ? fabsf(rsub(lv[i], left_level)) : __int_as_float(0x7f800000);
            rv[i] = e < count ? fabsf(rsub(rv[i], right_level)) : __int_as_float(0x7f800000);
        }
        reg_merge<G, V>(g, lv);
        reg_merge<G, V>(g, rv);
        store_run<G, V>(g, lv, scratch);
        store_run<G, V>(g, rv, scratch + N);
        g.sync();
        noise_median = union_median(scratch, scratch + N, count);
        g.sync();
    } else {
        // Edge medians (initial_guess.hpp:142-150) with shared-memory sorts.
        const int n1_mask = n1 - 1;
        for (int t = int(g.lane); t < 2 * n1; t += G) {
            const int j = t & n1_mask;
            scratch[t] = j < count ? ys[t >= n1 ? m - count + j : j] : __int_as_float(0x7f800000);
        }
        g.sync();
        bitonic_sort(g, scratch, n1, 2);
        left_level = sorted_median(scratch, count);
        right_level = sorted_median(scratch + n1, count);
        g.sync();
        // Union of both sorted sides: reverse the right run to make one bitonic sequence.
        for (int t = int(g.lane); t < n1 / 2; t += G) {
            const float a = scratch[n1 + t], b = scratch[2 * n1 - 1 - t];
            scratch[n1 + t] = b;
            scratch[2 * n1 - 1 - t] = a;
        }
        g.sync();
        bitonic_merge(g, scratch, 2 * n1);
        baseline = sorted_median(scratch, 2 * count);
        g.sync();
        slope = paired ? rdiv(rsub(right_level, left_level), rsub(xc.right_x, xc.left_x)) : 0.0f;
        level = paired ? left_level : baseline;
        // Absolute edge deviations (initial_guess.hpp:163-167), both sides sorted together.
        for (int t = int(g.lane); t < 2 * n1; t += G) {
            float v = __int_as_float(0x7f800000);
            if (t < count)
                v = fabsf(rsub(ys[t], left_level));
            else if (t >= n1 && t - n1 < count)
                v = fabsf(rsub(ys[m - count + (t - n1)], right_level));
            scratch[t] = v;
        }
        g.sync();
        bitonic_sort(g, scratch, 2 * n1, 1);
        noise_median = sorted_median(scratch, 2 * count);
        g.sync();
    }
    if (!isfinite(slope))
        return kGuessInvalid;
    // Noise scale: 1.4826 * median of absolute edge deviations (initial_guess.hpp:163-169).
    const float noise = rmul(1.4826f, noise_median);
    if (!isfinite(noise))
        return kGuessInvalid;
    // PRE: ys is this group's own staged, 16-byte aligned copy of the row (padded to
    // a multiple of 4 floats, as is xs).  The two-Lorentzian's signal needs x and is
    // read many times by the second-peak search: it overwrites the row once.  The
    // other models' signal is y - level, formed wherever a sample is read.
    constexpr bool overwrite = PRE && paired;
    if constexpr (overwrite) {
        const Signal<MODEL> raw{xs, ys, level, slope, xc.left_x, m};
        float4 *row = reinterpret_cast<float4 *>(const_cast<float *>(ys));
        const float4 *xq = reinterpret_cast<const float4 *>(xs);
        for (int q = int(g.lane); 4 * q < m; q += G) {
            const float4 yv = row[q];
            const float4 xv = paired ? xq[q] : yv; // x matters only with a slope
            row[q] = make_float4(raw.raw(yv.x, xv.x), raw.raw(yv.y, xv.y), raw.raw(yv.z, xv.z),
                                 raw.raw(yv.w, xv.w));
        }
        g.sync();
    }
    const Signal<MODEL, overwrite> s{xs, ys, level, slope, xc.left_x, m};
    // Tallest smoothed local maximum (initial_guess.hpp:170-179).  The same sweep
    // checks that every signal sample is finite (initial_guess.hpp:158-162); both
    // failures end in invalid_input, so their order does not matter.  For the
    // two-Lorentzian it also records every positive smoothed local maximum, the
    // candidates of the second-peak search, as bits of the lane (bit 4k+t of
    // lane l is sample 4(l + kG) - 2 + t; words stored word-major after the block
    // extrema in `scratch`).
    float height = 0.0f;
    int first = m;
    [[maybe_unused]] unsigned *cand_bits = reinterpret_cast<unsigned *>(scratch + 4 * walk_blocks(m));
    const bool signal_finite =
        chunk_sweep<G, paired, !overwrite, PRE>(g, s, ys, m, level, height, first, cand_bits);
    if (!g.all(signal_finite))
        return kGuessInvalid;
    argmax_pair(g, height, first);
    if (first == m || height <= rmul(3.0f, noise))
        return kGuessNoPeak;
    first = s.raw_maximum(first);
    PeakFeature primary = find_peak<G>(g, s, xs, first, 0, m - 1, false);
    if (!primary.valid)
        return kGuessNoPeak;
    if constexpr (!paired) {
        out[0] = primary.amplitude;
        out[1] = primary.center;
        if constexpr (MODEL == kGaussian)
            out[2] = rdiv(primary.width, 2.354820045030949382f);
        else if constexpr (MODEL == kLorentzian)
            out[2] = rhalf(primary.width);
        else {
            out[2] = primary.width;
            out[3] = 0.5f;
        }
    } else {
        // Second peak (initial_guess.hpp:199-227): the tallest smoothed local maximum
        // (ties: smaller index) that is far enough from the first and prominent
        // enough.  The candidates are the positive smoothed local maxima the first
        // sweep recorded (bits per lane).  One walk over each lane's candidates
        // collects its two best far-enough ones.  The best of the lanes' second
        // candidates is a cut-off: every candidate better than it is some lane's
        // first, so the candidates at or above the cut-off are the true leaders.
        // Each lane tests its own leaders; the best passing one is the answer.  When
        // all fail, the lanes test every candidate below the cut-off and keep the
        // best passing one.
        const float separation =
            smax(rmul(3.0f, xc.guess_spacing), rmul(2.0f, smin(primary.left_radius, primary.right_radius)));
        const float threshold = rmul(3.0f, noise);
        // The edge runs are no longer needed: their buffer holds the block extrema
        // (the candidate bits follow them).
        const int blocks = walk_blocks(m);
        float *bmin = scratch, *bmax = bmin + blocks, *pmin = bmax + blocks, *smin = pmin + blocks;
        block_extrema<G>(g, s, bmin, bmax);
        auto far_enough = [&](int j) {
            const int idx = s.raw_maximum(j);
            const int bins = idx > first ? idx - first : first - idx;
            return !(bins < 3 || fabsf(rsub(xs[idx], primary.center)) < separation);
        };
        const int words = chunk_words(m, G);
        auto cand_sample = [&](int b) { return chunk_sample(int(g.lane), b, G); };
        const unsigned *bits = cand_bits + int(g.lane);
        int second = m;
        float v1 = 0.0f, v2 = 0.0f;
        int j1 = m, j2 = m;
        for (int w = 0; w < words; ++w) {
            unsigned cand = bits[w * G];
            while (cand) {
                const int j = cand_sample(w * 32 + __ffs(cand) - 1);
                cand &= cand - 1;
                const float v = s.smooth_interior(j);
                if (!(v > v2 || (v == v2 && j < j2)) || !far_enough(j))
                    continue;
                if (v > v1 || (v == v1 && j < j1)) {
                    v2 = v1;
                    j2 = j1;
                    v1 = v;
                    j1 = j;
                } else {
                    v2 = v;
                    j2 = j;
                }
            }
        }
        float cut_v = v2;
        int cut_j = j2;
        argmax_pair(g, cut_v, cut_j); // cut_j == m: every candidate was collected
        auto leader = [&](float v, int j) {
            return j != m && (cut_j == m || v > cut_v || (v == cut_v && j <= cut_j));
        };
        const bool pass1 = leader(v1, j1) && may_be_prominent(pmin, smin, m, j1, v1, threshold) &&
                           prominent(s, bmin, bmax, j1, threshold);
        const bool pass2 = !pass1 && leader(v2, j2) && may_be_prominent(pmin, smin, m, j2, v2, threshold) &&
                           prominent(s, bmin, bmax, j2, threshold);
        float bv = pass1 ? v1 : pass2 ? v2 : 0.0f;
        int bj = pass1 ? j1 : pass2 ? j2 : m;
        argmax_pair(g, bv, bj);
        if (bj == m && cut_j != m) {
            // Every candidate below the cut-off, each lane its own (its samples are
            // 1+l, 1+l+G, ...: candidates cluster on the peaks, and interleaving
            // spreads them over the lanes).  A lane takes one step per loop turn -- a
            // candidate check or one step of a prominence walk (the walks of
            // prominent(), unrolled, sliding a window over the signal: one new sample
            // per step) -- so the lanes' walks run side by side instead of each turn
            // waiting for the longest.
            auto smooth3 = [](float a, float b, float c) {
                return radd(radd(rmul(0.25f, a), rmul(0.5f, b)), rmul(0.25f, c));
            };
            int cw = -1;
            unsigned cand = 0;
            int j = m;
            int walk = 0; // 0: checking candidates, -1 / +1: walking left / right of j
            int w = 0;
            float h = 0.0f, wo = 0.0f, wi = 0.0f; // walk window: at(w), at(w -/+ 1 towards j)
            bool fresh = true;
            while (true) {
                if (walk == 0) {
                    while (cand == 0 && cw + 1 < words)
                        cand = bits[++cw * G];
                    if (cand == 0)
                        break;
                    j = cand_sample(cw * 32 + __ffs(cand) - 1);
                    cand &= cand - 1;
                    const float v = s.smooth_interior(j);
                    if ((v < cut_v || (v == cut_v && j > cut_j)) && (v > bv || (v == bv && j < bj)) &&
                        may_be_prominent(pmin, smin, m, j, v, threshold) && far_enough(j)) {
                        walk = -1;
                        w = j - 1;
                        h = v;
                        fresh = true;
                    }
                    continue;
                }
                // One step of the walk in direction `walk` (both directions share this
                // code, so the lanes of a warp do not split three ways).  The window
                // keeps wo = at(w) and wi = at(w - walk); smoothing sums s[w-1],
                // s[w], s[w+1] in that order, as detail::smooth does.
                bool fail = false, clear = false;
                const int edge = walk < 0 ? 0 : m - 1; // no smoothing at the ends
                if (walk < 0 ? w < 0 : w >= m) {
                    fail = true;
                } else if ((w & (kWalkBlock - 1)) == (walk < 0 ? kWalkBlock - 1 : 0) && bmax[w / kWalkBlock] <= h) {
                    clear = rsub(h, bmin[w / kWalkBlock]) > threshold;
                    w += walk * kWalkBlock;
                    fresh = true;
                } else {
                    if (fresh) {
                        wo = s.at(w);
                        wi = s.at(w - walk);
                        fresh = false;
                    }
                    float outer = 0.0f, v = wo;
                    if (w != edge) {
                        outer = s.at(w + walk);
                        v = walk < 0 ? smooth3(outer, wo, wi) : smooth3(wi, wo, outer);
                    }
                    fail = v > h;
                    clear = !fail && rsub(h, v) > threshold;
                    wi = wo;
                    wo = outer;
                    w += walk;
                }
                if (clear) {
                    if (walk < 0) { // left side clears: walk right
                        walk = 1;
                        w = j + 1;
                        fresh = true;
                        continue;
                    }
                    bv = h; // both sides clear: the lane's best so far
                    bj = j;
                    fail = true;
                }
                if (fail)
                    walk = 0;
            }
            argmax_pair(g, bv, bj);
        }
        if (bj != m)
            second = s.raw_maximum(bj);
        if (second == m)
            return kGuessInsufficient;
        if (first > second) {
            const int t = first;
            first = second;
            second = t;
        }
        // First minimum of signal[first+1 .. second-1].
        float mv = __int_as_float(0x7f800000);
        int mi = second;
        for (int j = first + 1 + int(g.lane); j < second; j += G) {
            const float v = s.at(j);
            if (v < mv) {
                mv = v;
                mi = j;
            }
        }
#pragma unroll
        for (int o = G / 2; o >= 1; o >>= 1) {
            const float ov = g.xor_(mv, o);
            const int oi = g.xor_(mi, o);
            if (ov < mv || (ov == mv && oi < mi)) {
                mv = ov;
                mi = oi;
            }
        }
        const int valley = mi;
        primary = find_peak<G>(g, s, xs, first, 0, valley, true);
        const PeakFeature secondary = find_peak<G>(g, s, xs, second, valley, m - 1, true);
        if (!primary.valid || !secondary.valid || !(primary.center < secondary.center))
            return kGuessInsufficient;
        out[0] = primary.amplitude;
        out[1] = primary.center;
        out[2] = rhalf(primary.width);
        out[3] = secondary.amplitude;
        out[4] = secondary.center;
        out[5] = rhalf(secondary.width);
        out[6] = rsub(left_level, rmul(slope, xc.left_x));
        out[7] = slope;
    }
#pragma unroll
    for (int k = 0; k < P; ++k)
        if (!isfinite(out[k]))
            return kGuessInvalid;
    if (!(out[2] > 0.0f) || (paired && !(out[5] > 0.0f)))
        return kGuessInvalid;
    return kGuessSuccess;
}

} // namespace bf
