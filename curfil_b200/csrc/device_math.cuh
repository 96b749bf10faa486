// Device restatement of CURFIL's depth-scaled two-box feature (random_tree_image.h:82-87,
// 222-316, 485-623; random_tree_image_gpu.cu:76-213) and of the normalised information-gain
// score (score.h:45-216).
//
// Floating-point operations are written with explicit round-to-nearest intrinsics so that the
// compiler cannot contract them into FMAs: every response is bit-identical to the host
// reference's double computation, and the scores differ from it only by the log2
// implementation.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cf {

constexpr int kDepthFeature = 0;
constexpr int kColorFeature = 1;

// Integral images of one dataset in device memory.
struct DsView {
    const float* color;   // [n][3][H][W]
    const int2* depth;    // [n][H][W] {sum mm (wrapping int32), valid count}
    int n, width, height;
    long long plane;      // W * H
};

// cf_sample in device code.
struct __align__(16) Sample {
    uint16_t x, y;
    uint32_t image;
    float depth;
    uint8_t label;
    uint8_t flip;
    uint16_t reserved;
};

// One candidate feature, unpacked from the int8 [11][F] table.
struct FeatParams {
    int8_t o1x, o1y, o2x, o2y, r1x, r1y, r2x, r2y;
    uint8_t type, ch1, ch2, pad;
};

__device__ __forceinline__ double dnan() { return __longlong_as_double(0x7ff8000000000000ULL); }

// XY::normalize: int / float -> float division, truncation toward zero.
__device__ __forceinline__ int norm_coord(int v, float depth) {
    return __float2int_rz(__fdiv_rn(static_cast<float>(v), depth));
}

// PixelInstance::averageRegionDepth; (x, y) already offset, (w, h) already max(1, .)
__device__ __forceinline__ double region_depth(const DsView& ds, uint32_t img, int x, int y, int w, int h) {
    const int lx = x - w, rx = x + w, uy = y - h, ly = y + h;
    if (lx < 0 || rx >= ds.width || uy < 0 || ly >= ds.height) return dnan();
    const int2* D = ds.depth + static_cast<long long>(img) * ds.plane;
    const int2 ul = __ldg(D + static_cast<long long>(uy) * ds.width + lx);
    const int2 ur = __ldg(D + static_cast<long long>(uy) * ds.width + rx);
    const int2 ll = __ldg(D + static_cast<long long>(ly) * ds.width + lx);
    const int2 lr = __ldg(D + static_cast<long long>(ly) * ds.width + rx);
    const int numValid = (lr.y - ur.y) + (ul.y - ll.y);
    if (numValid == 0) return dnan();
    // exact box sum: the wrapped 32-bit integrals differ by less than 2^31 inside one box
    const int sum = static_cast<int>((static_cast<uint32_t>(lr.x) - static_cast<uint32_t>(ur.x)) +
                                     (static_cast<uint32_t>(ul.x) - static_cast<uint32_t>(ll.x)));
    const double feat = __ddiv_rn(static_cast<double>(sum), 1000.0);
    return __ddiv_rn(feat, static_cast<double>(numValid));
}

// PixelInstance::averageRegionColor
__device__ __forceinline__ double region_color(const DsView& ds, uint32_t img, int ch, int x, int y, int w, int h) {
    const int lx = x - w, rx = x + w, uy = y - h, ly = y + h;
    if (lx < 0 || rx >= ds.width || uy < 0 || ly >= ds.height) return dnan();
    const float* P = ds.color + (static_cast<long long>(img) * 3 + ch) * ds.plane;
    const double lr = __ldg(P + static_cast<long long>(ly) * ds.width + rx);
    const double ll = __ldg(P + static_cast<long long>(ly) * ds.width + lx);
    const double ur = __ldg(P + static_cast<long long>(uy) * ds.width + rx);
    const double ul = __ldg(P + static_cast<long long>(uy) * ds.width + lx);
    if (isnan(lr) || isnan(ll) || isnan(ur) || isnan(ul)) return dnan();
    return __dadd_rn(__dsub_rn(lr, ur), __dsub_rn(ul, ll));
}

// ImageFeatureFunction::calculateFeatureResponse for a pixel at (px, py) with depth `depth`.
__device__ __forceinline__ double feature_response(const DsView& ds, uint32_t img, int px, int py, float depth,
                                                   const FeatParams& f, bool flip) {
    if (!(depth > 0.0f)) return dnan();
    const int o1x = flip ? -f.o1x : f.o1x;
    const int o2x = flip ? -f.o2x : f.o2x;
    const int w1 = max(1, norm_coord(f.r1x, depth)), h1 = max(1, norm_coord(f.r1y, depth));
    const int x1 = px + norm_coord(o1x, depth), y1 = py + norm_coord(f.o1y, depth);
    double a;
    if (f.type == kDepthFeature)
        a = region_depth(ds, img, x1, y1, w1, h1);
    else
        a = region_color(ds, img, f.ch1, x1, y1, w1, h1);
    if (isnan(a)) return a;
    const int w2 = max(1, norm_coord(f.r2x, depth)), h2 = max(1, norm_coord(f.r2y, depth));
    const int x2 = px + norm_coord(o2x, depth), y2 = py + norm_coord(f.o2y, depth);
    double b;
    if (f.type == kDepthFeature)
        b = region_depth(ds, img, x2, y2, w2, h2);
    else
        b = region_color(ds, img, f.ch2, x2, y2, w2, h2);
    if (isnan(b)) return b;
    return __dsub_rn(a, b);
}

__device__ __forceinline__ double sample_response(const DsView& ds, const Sample& s, const FeatParams& f, bool flip) {
    return feature_response(ds, s.image, s.x, s.y, s.depth, f, flip);
}

__device__ __forceinline__ FeatParams load_feature(const int8_t* table, int F, int f) {
    FeatParams p;
    p.type = static_cast<uint8_t>(table[f]);
    p.o1x = table[1 * F + f];
    p.o1y = table[2 * F + f];
    p.o2x = table[3 * F + f];
    p.o2y = table[4 * F + f];
    p.r1x = table[5 * F + f];
    p.r1y = table[6 * F + f];
    p.r2x = table[7 * F + f];
    p.r2y = table[8 * F + f];
    p.ch1 = static_cast<uint8_t>(table[9 * F + f]);
    p.ch2 = static_cast<uint8_t>(table[10 * F + f]);
    p.pad = 0;
    return p;
}

// ---- normalised information gain (score.h) -------------------------------------------------

__device__ __forceinline__ double entropy_of(double p) {
    return p == 0.0 ? 0.0 : __dmul_rn(-p, log2(p));
}

__device__ __forceinline__ double normalize_score(double s) {
    if (s > 1.0) return 1.0;
    if (s < 0.0) return 0.0;
    return s;
}

// Classification entropy H_c of a node (score.h:174-189), classes in ascending label order.
static __device__ __noinline__ double classification_entropy(int num_present, const uint32_t* present_counts, double total) {
    double hc = 0;
    for (int i = 0; i < num_present; i++) hc = __dadd_rn(hc, entropy_of(static_cast<double>(present_counts[i])));
    hc = __dsub_rn(hc, entropy_of(total));
    return __ddiv_rn(hc, total);
}

// One term of InformationGainScore::calculateScore (score.h:118-128).
__device__ __forceinline__ double ig_term(double value, double total, double sideProb, double classProb) {
    const double p = __ddiv_rn(value, total);
    return __dmul_rn(p, log2(__ddiv_rn(p, __dmul_rn(sideProb, classProb))));
}

// ---- float bounds of the score (screening) ----------------------------------------------------
// With f(x) = x log2 x, the score of a split with left counts l_i, right counts r_i = h_i - l_i,
// L = sum l_i, R = sum r_i, node total N is, in real arithmetic,
//     score = 2 S / D,  S = sum f(l_i) + sum f(r_i) - f(L) - f(R) + K,  D = f(N) - f(L) - f(R) + K,
// K = f(N) - sum f(h_i)  (S = N * information gain, D = N * (H_split + H_classes)).
// score_bounds evaluates S and D in 2^23-scaled fixed point (below) and widens them by a bound on
// the log2 error, so the reference's double score lies in [lb, ub]; the widening is far above the
// rounding error of the reference's own double evaluation. Where D may be tiny relative to N the
// bounds are [0, 1].
struct ScoreConsts {
    double fN;      // f(N)
    double K;       // f(N) - sum f(h_i)
    double Nd;      // N
    uint32_t N;
};

// round(2^23 x log2 x) up to x (2^-22 + 2^-23) 2^23: with float(x) = m 2^e, m in [1, 2),
// x log2 x ~ x (e + log2 m); e is exact, __log2f(m) has absolute error <= 2^-22 on [1, 2], its 23
// fraction bits are rounded (2^-24) and float(x) is rounded for x > 2^24 (x log2(1 + 2^-24) <
// 1.5 x 2^-24). The product x * (e 2^23 + frac) < 2^60 is exact in 64-bit integers, so sums of
// these terms carry no rounding error at all.
__device__ __forceinline__ long long xlog2x_fixed(uint32_t x) {
    const uint32_t b = __float_as_uint(__uint2float_rn(x));
    const uint32_t e = (b >> 23) - 127u;
    const float lg = fmaxf(__log2f(__uint_as_float((b & 0x7FFFFFu) | 0x3F800000u)), 0.0f);
    const uint32_t frac = __float_as_uint(lg + 1.0f) - 0x3F800000u;   // round(2^23 lg), <= 2^23
    const unsigned long long p = static_cast<unsigned long long>(x) * ((e << 23) + frac);
    return x == 0u ? 0LL : static_cast<long long>(p);
}

__device__ __forceinline__ ScoreConsts score_consts(const uint32_t* counts, int n) {
    double N = 0, sum_fh = 0;
    for (int i = 0; i < n; i++) {
        const double h = static_cast<double>(counts[i]);
        N += h;
        if (h > 0) sum_fh += h * log2(h);
    }
    ScoreConsts k;
    k.fN = N > 0 ? N * log2(N) : 0.0;
    k.K = k.fN - sum_fh;
    k.Nd = N;
    k.N = static_cast<uint32_t>(N);
    return k;
}

// (lb, ub) of the score; left(i) = left count of class i (i < n), counts[i] = h_i.
template <typename LeftCount>
__device__ __forceinline__ float2 score_bounds(LeftCount left, const uint32_t* counts, int n, const ScoreConsts& k) {
    uint32_t L = 0;
    long long acc = 0;
    for (int i = 0; i < n; i++) {
        const uint32_t l = left(i);
        L += l;
        acc += xlog2x_fixed(l) + xlog2x_fixed(counts[i] - l);
    }
    const uint32_t R = k.N - L;
    if (L == 0u || R == 0u) return make_float2(0.0f, 0.0f);   // the reference scores 0
    const long long fLR = xlog2x_fixed(L) + xlog2x_fixed(R);
    const double S = static_cast<double>(acc - fLR) * 0x1p-23 + k.K;    // N * information gain
    const double D = k.fN - static_cast<double>(fLR) * 0x1p-23 + k.K;   // N * (H_split + H_classes)
    // every x of the sum of l_i, r_i terms (2N in total) and of L, R (N) contributes
    // <= 0.75 x 2^-21; 2^-19 N covers S and D with room for the products' and sums' roundings
    const double e = 0x1p-19 * k.Nd;
    const float dlo = static_cast<float>(D - e);
    if (!(dlo > 1e-4f * static_cast<float>(k.Nd))) return make_float2(0.0f, 1.0f);
    float ub = 2.0f * static_cast<float>(S + e) / dlo;
    float lb = 2.0f * static_cast<float>(S - e) / static_cast<float>(D + e);
    ub = fminf(1.0f, fmaxf(0.0f, ub * 1.0000038f + 1e-8f));   // (1 + 2^-18), covers the float ops above
    lb = fminf(1.0f, fmaxf(0.0f, lb * 0.9999962f - 1e-8f));
    return make_float2(lb, ub);
}

}  // namespace cf
