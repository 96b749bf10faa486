// Threshold bin of one feature response, computed with fast paths that fall back to the exact
// reference arithmetic whenever the fast result could differ. The bin (number of thresholds the
// response exceeds) is therefore always identical to the one obtained from the exact double
// response of random_tree_image.h:564-623.
//
// 1. Depth-scaled offsets: the reference computes trunc(RN(v / d)) for integer v and float d > 0.
//    q = RN(|v| * RN(1/d)) and y = RN(|v|/d) both lie within q (1 +- 2^-22). lo = RD(q (1 - 2^-21))
//    and hi = RU(q (1 + 2^-21)) bracket y; when floor(lo) == floor(hi) that is floor(y), so
//    trunc(RN(v/d)) = sign(v) * floor(lo). Otherwise the correctly rounded division is evaluated.
//    floor() of a value in [0, 2^23) is taken on the FMA pipe: RD(x + 2^23) = 2^23 + floor(x).
//    (d >= 0.001 because pixel depths are integer millimetres, so q <= 127000 < 2^23.)
// 2. Depth features: a = RN(RN(sum/1000)/n) per box. The float estimate fdividef(sum, n) * 0.001f
//    is within 7 * 2^-24 relative of a (int->float 2^-24, fdividef 2 ulp, constant and product
//    2^-24 each), so r' = a' - b' is within 4.8e-7 (|a| + |b|) of the exact response r. With
//    delta = 2e-6 (|a'| + |b'|): if no threshold lies in [r' - delta, r' + delta], every threshold
//    compares the same against r and r', and the bin is #{t < r' - delta}. Otherwise the two
//    double divisions of the reference are evaluated and the exact response is binned.
// 3. Colour features are evaluated exactly (integer-valued float corners summed in double).
// NaN responses (box outside the image, no valid depth in a box, invalid pixel depth) depend only
// on integer tests and land in bin T (right of every threshold, `!(r <= t)`).
#pragma once

#include "device_math.cuh"

namespace cf {

struct EvalPixel {
    const float* color;   // colour integral of the sample's image, [3][H][W]
    const int2* depth;    // depth integral of the sample's image, [H][W]
    int x, y;
    float d, inv_d;       // depth in metres and RN(1/d); d <= 0 marks an invalid pixel depth
};

__device__ __forceinline__ EvalPixel make_eval_pixel(const DsView& ds, const Sample& s) {
    EvalPixel p;
    p.color = ds.color + static_cast<long long>(s.image) * 3 * ds.plane;
    p.depth = ds.depth + static_cast<long long>(s.image) * ds.plane;
    p.x = s.x;
    p.y = s.y;
    p.d = s.depth;
    p.inv_d = s.depth > 0.0f ? __frcp_rn(s.depth) : 0.0f;
    return p;
}

// Slow paths, kept out of line so their registers do not weigh on the hot loop.
static __device__ __noinline__ int exact_norm_abs(float av, float d) { return __float2int_rz(__fdiv_rn(av, d)); }

// trunc(RN(v / d)) of XY::normalize; av = |v| as float (0 gives 0 without a special case)
__device__ __forceinline__ int fast_norm(int v, float av, float d, float inv_d) {
    const float q = __fmul_rn(av, inv_d);
    const float lo = __fmaf_rd(q, -4.76837158203125e-07f, q);   // q (1 - 2^-21), rounded down
    const float hi = __fmaf_ru(q, 4.76837158203125e-07f, q);    // q (1 + 2^-21), rounded up
    const float tl = __fadd_rd(lo, 8388608.0f);                 // 2^23 + floor(lo)
    const float th = __fadd_rd(hi, 8388608.0f);
    int r = __float_as_int(tl) - 0x4B000000;
    if (tl != th) r = exact_norm_abs(av, d);
    return v < 0 ? -r : r;
}

// Two fast_norm evaluations in packed f32x2 arithmetic (sm_100): the same operations and roundings
// per value as fast_norm, two values per instruction.
__device__ __forceinline__ unsigned long long pack_f2(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void unpack_f2(unsigned long long v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ void fast_norm2(int v0, int v1, float av0, float av1, float d, float inv_d, int& r0,
                                           int& r1) {
    const unsigned long long a = pack_f2(av0, av1), inv = pack_f2(inv_d, inv_d);
    const unsigned long long em = pack_f2(-4.76837158203125e-07f, -4.76837158203125e-07f);
    const unsigned long long ep = pack_f2(4.76837158203125e-07f, 4.76837158203125e-07f);
    const unsigned long long big = pack_f2(8388608.0f, 8388608.0f);
    unsigned long long q, lo, hi, tl, th;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(q) : "l"(a), "l"(inv));
    asm("fma.rm.f32x2 %0, %1, %2, %1;" : "=l"(lo) : "l"(q), "l"(em));   // q (1 - 2^-21), rounded down
    asm("fma.rp.f32x2 %0, %1, %2, %1;" : "=l"(hi) : "l"(q), "l"(ep));   // q (1 + 2^-21), rounded up
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(tl) : "l"(lo), "l"(big));     // 2^23 + floor(lo)
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(th) : "l"(hi), "l"(big));
    float tl0, tl1, th0, th1;
    unpack_f2(tl, tl0, tl1);
    unpack_f2(th, th0, th1);
    int a0 = __float_as_int(tl0) - 0x4B000000, a1 = __float_as_int(tl1) - 0x4B000000;
    if (tl0 != th0) a0 = exact_norm_abs(av0, d);
    if (tl1 != th1) a1 = exact_norm_abs(av1, d);
    r0 = v0 < 0 ? -a0 : a0;
    r1 = v1 < 0 ? -a1 : a1;
}

// Normalisation policies of feature_bin.
// CheckedNorm: fast_norm, each value checked on its own; pair() scales two values at once.
struct CheckedNorm {
    __device__ __forceinline__ int operator()(int v, float av, float d, float inv_d) const {
        return fast_norm(v, av, d, inv_d);
    }
    __device__ __forceinline__ void pair(int v0, int v1, float av0, float av1, float d, float inv_d, int& r0,
                                         int& r1) const {
        fast_norm2(v0, v1, av0, av1, d, inv_d, r0, r1);
    }
};

// trunc(RN(v / d)) for an int parameter (used outside the hot loop)
__device__ __forceinline__ int fast_norm(int v, float d, float inv_d) {
    return fast_norm(v, static_cast<float>(v < 0 ? -v : v), d, inv_d);
}

// A candidate feature prepared for the hot loop: the eight parameters and their magnitudes as
// floats (no int->float conversion per evaluation).
struct __align__(16) EvalFeat {
    float av[8];          // |o1x|, |o1y|, |o2x|, |o2y|, |r1x|, |r1y|, |r2x|, |r2y|
    int8_t v[8];          // o1x, o1y, o2x, o2y, r1x, r1y, r2x, r2y
    uint8_t type, ch1, ch2, pad;
    uint32_t pad2[3];
};

__device__ __forceinline__ EvalFeat make_eval_feat(const FeatParams& f) {
    EvalFeat e;
    const int8_t v[8] = {f.o1x, f.o1y, f.o2x, f.o2y, f.r1x, f.r1y, f.r2x, f.r2y};
#pragma unroll
    for (int i = 0; i < 8; i++) {
        e.v[i] = v[i];
        // |v| <= 128 converts exactly through the float bit pattern of 2^23 + |v|
        e.av[i] = __fsub_rn(__int_as_float(0x4B000000 | (v[i] < 0 ? -v[i] : v[i])), 8388608.0f);
    }
    e.type = f.type;
    e.ch1 = f.ch1;
    e.ch2 = f.ch2;
    e.pad = 0;
    e.pad2[0] = e.pad2[1] = e.pad2[2] = 0;
    return e;
}

// Thresholds of one feature in shared memory: sorted ascending. With kPad = 32 (T <= 31) or 64
// (32 <= T <= 63) the row has kPad entries, positions T..kPad-1 holding +inf, and is searched
// branch-free in five or six steps; kPad = 0 keeps the T thresholds and a binary search. (Five steps
// give 32 outcomes, counts 0..31, so a row of 32 serves T <= 31 only.)
constexpr int kPadThresholds = 32;

// the padded row width for T thresholds (0: no padding)
__host__ __device__ constexpr int padded_row(int T) { return T < 32 ? 32 : (T < 64 ? 64 : 0); }

// #{i : sorted[i] < v}
template <int kPad>
__device__ __forceinline__ int count_below(const float* sorted, int T, float v) {
    if (kPad == 64) {
        int k = sorted[31] < v ? 32 : 0;
        k += sorted[k + 15] < v ? 16 : 0;
        k += sorted[k + 7] < v ? 8 : 0;
        k += sorted[k + 3] < v ? 4 : 0;
        k += sorted[k + 1] < v ? 2 : 0;
        k += sorted[k] < v ? 1 : 0;
        return k;
    }
    if (kPad == 32) {
        int k = sorted[15] < v ? 16 : 0;
        k += sorted[k + 7] < v ? 8 : 0;
        k += sorted[k + 3] < v ? 4 : 0;
        k += sorted[k + 1] < v ? 2 : 0;
        k += sorted[k] < v ? 1 : 0;
        return k;
    }
    int lo = 0, n = T;
    while (n > 0) {
        const int half = n >> 1;
        if (sorted[lo + half] < v) {
            lo += half + 1;
            n -= half + 1;
        } else {
            n = half;
        }
    }
    return lo;
}

// bin of an exact double response: #{t : !(r <= t)}; r <= t (float t) iff RU(r) <= t
template <int kPad>
__device__ __forceinline__ int exact_bin(double r, const float* sorted, int T) {
    if (isnan(r)) return T;
    return count_below<kPad>(sorted, T, __double2float_ru(r));
}

// exact depth response ((s1/1000)/n1 - (s2/1000)/n2 in double, random_tree_image.h:313-315)
static __device__ __noinline__ double exact_depth_response(int s1, int nv1, int s2, int nv2) {
    const double A = __ddiv_rn(__ddiv_rn(static_cast<double>(s1), 1000.0), static_cast<double>(nv1));
    const double B = __ddiv_rn(__ddiv_rn(static_cast<double>(s2), 1000.0), static_cast<double>(nv2));
    return __dsub_rn(A, B);
}

// Binning policies of feature_bin.
// SortedBins: the number of a feature's sorted thresholds t with !(r <= t) (0..T; NaN -> T).
template <int kPad>
struct SortedBins {
    const float* sorted;
    int T;
    __device__ __forceinline__ int nan() const { return T; }
    // bin of every r in [r0 - delta, r0 + delta] if it is the same for all of them
    __device__ __forceinline__ bool fast(float r0, float delta, int& k) const {
        k = count_below<kPad>(sorted, T, r0 - delta);
        return k == T || sorted[k] > r0 + delta;   // k == T: no threshold above, sorted[T] may lie past the row
    }
    __device__ __forceinline__ int exact(double r) const { return exact_bin<kPad>(r, sorted, T); }
};

// ThresholdSide: 1 when the sample goes right of one split, !(r <= threshold) (NaN goes right).
struct ThresholdSide {
    float thr;
    __device__ __forceinline__ int nan() const { return 1; }
    __device__ __forceinline__ bool fast(float r0, float delta, int& k) const {
        k = r0 - delta > thr ? 1 : 0;
        return r0 - delta > thr || r0 + delta < thr;
    }
    __device__ __forceinline__ int exact(double r) const { return r <= static_cast<double>(thr) ? 0 : 1; }
};

template <typename Bins, typename Norm = CheckedNorm>
__device__ __forceinline__ int feature_bin(const EvalPixel& p, int W, int H, const EvalFeat& f, bool flip,
                                           const Bins& bins, const Norm& norm = Norm()) {
    const int T = bins.nan();
    if (!(p.d > 0.0f)) return T;
    const int o1x = flip ? -f.v[0] : f.v[0];
    const int o2x = flip ? -f.v[2] : f.v[2];
    int nx1, ny1, nw1, nh1;
    norm.pair(o1x, f.v[1], f.av[0], f.av[1], p.d, p.inv_d, nx1, ny1);
    norm.pair(f.v[4], f.v[5], f.av[4], f.av[5], p.d, p.inv_d, nw1, nh1);
    const int x1 = p.x + nx1, y1 = p.y + ny1, w1 = max(1, nw1), h1 = max(1, nh1);
    if (x1 - w1 < 0 || x1 + w1 >= W || y1 - h1 < 0 || y1 + h1 >= H) return T;
    int nx2, ny2, nw2, nh2;
    norm.pair(o2x, f.v[3], f.av[2], f.av[3], p.d, p.inv_d, nx2, ny2);
    norm.pair(f.v[6], f.v[7], f.av[6], f.av[7], p.d, p.inv_d, nw2, nh2);
    const int x2 = p.x + nx2, y2 = p.y + ny2, w2 = max(1, nw2), h2 = max(1, nh2);
    if (x2 - w2 < 0 || x2 + w2 >= W || y2 - h2 < 0 || y2 + h2 >= H) return T;
    const int ul1 = (y1 - h1) * W + (x1 - w1), ur1 = (y1 - h1) * W + (x1 + w1);
    const int ll1 = (y1 + h1) * W + (x1 - w1), lr1 = (y1 + h1) * W + (x1 + w1);
    const int ul2 = (y2 - h2) * W + (x2 - w2), ur2 = (y2 - h2) * W + (x2 + w2);
    const int ll2 = (y2 + h2) * W + (x2 - w2), lr2 = (y2 + h2) * W + (x2 + w2);
    if (f.type == kDepthFeature) {
        const int2 a_ul = __ldg(p.depth + ul1), a_ur = __ldg(p.depth + ur1);
        const int2 a_ll = __ldg(p.depth + ll1), a_lr = __ldg(p.depth + lr1);
        const int2 b_ul = __ldg(p.depth + ul2), b_ur = __ldg(p.depth + ur2);
        const int2 b_ll = __ldg(p.depth + ll2), b_lr = __ldg(p.depth + lr2);
        const int nv1 = (a_lr.y - a_ur.y) + (a_ul.y - a_ll.y);
        const int nv2 = (b_lr.y - b_ur.y) + (b_ul.y - b_ll.y);
        if (nv1 == 0 || nv2 == 0) return T;
        const int s1 = static_cast<int>((static_cast<uint32_t>(a_lr.x) - static_cast<uint32_t>(a_ur.x)) +
                                        (static_cast<uint32_t>(a_ul.x) - static_cast<uint32_t>(a_ll.x)));
        const int s2 = static_cast<int>((static_cast<uint32_t>(b_lr.x) - static_cast<uint32_t>(b_ur.x)) +
                                        (static_cast<uint32_t>(b_ul.x) - static_cast<uint32_t>(b_ll.x)));
        // counts outside [1, 2^23): boxes of more than 2^23 pixels, or negative counts where a box
        // reaches the zero depth padding of a resized frame (the reference divides by them as they are)
        if (static_cast<uint32_t>(nv1 - 1) >= 0x7FFFFFu || static_cast<uint32_t>(nv2 - 1) >= 0x7FFFFFu)
            return bins.exact(exact_depth_response(s1, nv1, s2, nv2));
        // 1 <= nv < 2^23 (checked above) converts exactly through the float bit pattern (no conversion unit)
        const float n1f = __fsub_rn(__int_as_float(0x4B000000 + nv1), 8388608.0f);
        const float n2f = __fsub_rn(__int_as_float(0x4B000000 + nv2), 8388608.0f);
        const float a = __fdividef(static_cast<float>(s1), n1f) * 0.001f;
        const float b = __fdividef(static_cast<float>(s2), n2f) * 0.001f;
        const float r = a - b;
        const float delta = 2e-6f * (fabsf(a) + fabsf(b)) + 1e-30f;
        int k;
        if (bins.fast(r, delta, k)) return k;
        return bins.exact(exact_depth_response(s1, nv1, s2, nv2));
    }
    const float* P1 = p.color + static_cast<long long>(f.ch1) * W * H;
    const float* P2 = p.color + static_cast<long long>(f.ch2) * W * H;
    const float c_lr = __ldg(P1 + lr1), c_ur = __ldg(P1 + ur1), c_ul = __ldg(P1 + ul1), c_ll = __ldg(P1 + ll1);
    const float d_lr = __ldg(P2 + lr2), d_ur = __ldg(P2 + ur2), d_ul = __ldg(P2 + ul2), d_ll = __ldg(P2 + ll2);
    if (isnan(c_lr) || isnan(c_ur) || isnan(c_ul) || isnan(c_ll) || isnan(d_lr) || isnan(d_ur) || isnan(d_ul) ||
        isnan(d_ll))
        return T;
    const double A = __dadd_rn(__dsub_rn(static_cast<double>(c_lr), static_cast<double>(c_ur)),
                               __dsub_rn(static_cast<double>(c_ul), static_cast<double>(c_ll)));
    const double B = __dadd_rn(__dsub_rn(static_cast<double>(d_lr), static_cast<double>(d_ur)),
                               __dsub_rn(static_cast<double>(d_ul), static_cast<double>(d_ll)));
    return bins.exact(__dsub_rn(A, B));
}

// Feature parameters of a packed split node, prepared for feature_bin.
__device__ __forceinline__ EvalFeat eval_feat_of(int8_t o1x, int8_t o1y, int8_t o2x, int8_t o2y, int8_t r1x,
                                                 int8_t r1y, int8_t r2x, int8_t r2y, int type, int ch1, int ch2) {
    FeatParams fp;
    fp.o1x = o1x;
    fp.o1y = o1y;
    fp.o2x = o2x;
    fp.o2y = o2y;
    fp.r1x = r1x;
    fp.r1y = r1y;
    fp.r2x = r2x;
    fp.r2y = r2y;
    fp.type = static_cast<uint8_t>(type);
    fp.ch1 = static_cast<uint8_t>(ch1);
    fp.ch2 = static_cast<uint8_t>(ch2);
    fp.pad = 0;
    return make_eval_feat(fp);
}

}  // namespace cf
