// Candidate features of one tree level: generation, stable sort by getSortKey, and the
// per-feature threshold ranks used by the single-increment histogram.
//
// Generation follows generateRandomFeaturesKernel (random_tree_image_gpu.cu:250-390): one thread
// per candidate, feature type and channels fixed by the candidate index, offsets and regions
// drawn from a per-candidate stream, and each threshold the response of a random sample of the
// level (NaN mapped to 0). The cuRAND XORWOW stream is replaced by Philox4x32-10 (Salmon et al.,
// SC'11) keyed by (seed, candidate): the reference stream cannot be reproduced without
// cuRAND's skip-ahead tables, and Philox makes the host restatement exact.
#include "features.h"

namespace cf {

namespace {

constexpr int kMaxRedraws = 1000;

__device__ __forceinline__ void philox4x32_10(uint32_t k0, uint32_t k1, uint32_t c[4]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
        const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

struct Stream {
    uint32_t k0, k1, block, pos;
    uint32_t buf[4];
    __device__ Stream(uint32_t seed, uint32_t feat) : k0(seed), k1(feat), block(0), pos(4) {}
    __device__ uint32_t next() {
        if (pos == 4) {
            buf[0] = block++;
            buf[1] = buf[2] = buf[3] = 0;
            philox4x32_10(k0, k1, buf);
            pos = 0;
        }
        return buf[pos++];
    }
    // uniform in (0, 1], exact
    __device__ float uniform() { return __fmul_rn(__uint2float_rn((next() >> 8) + 1u), 1.0f / 16777216.0f); }
};

// randomOffset (random_tree_image_gpu.cu:226-238): u * 2 * (radius+1) - (radius+1), truncated
__device__ __forceinline__ int8_t draw_offset(Stream& s, float br) {
    float t = __fmul_rn(s.uniform(), 2.0f);
    t = __fmul_rn(t, br);
    t = __fsub_rn(t, br);
    return static_cast<int8_t>(__float2int_rz(t));
}

// randomRegion (random_tree_image_gpu.cu:240-248): u * regionSize + 1, truncated
__device__ __forceinline__ int8_t draw_region(Stream& s, float rs) {
    float t = __fmul_rn(s.uniform(), rs);
    t = __fadd_rn(t, 1.0f);
    return static_cast<int8_t>(__float2int_rz(t));
}

__global__ void __launch_bounds__(128)
gen_features_kernel(DsView ds, const Sample* __restrict__ samples, uint32_t num_samples, uint32_t seed, int F, int T,
                    int box_radius, int region_size, int use_depth, int8_t* __restrict__ raw_feat,
                    float* __restrict__ raw_thr, int32_t* __restrict__ keys) {
    const int feat = blockIdx.x * blockDim.x + threadIdx.x;
    if (feat >= F) return;
    Stream rng(seed, static_cast<uint32_t>(feat));
    const uint8_t type = use_depth ? static_cast<uint8_t>(feat >= F / 2) : 1;
    const float br = static_cast<float>(static_cast<uint8_t>(static_cast<uint8_t>(box_radius) + 1));
    const float rs = static_cast<float>(static_cast<uint8_t>(region_size));
    FeatParams p;
    p.type = type;
    p.o1x = draw_offset(rng, br);
    p.o1y = draw_offset(rng, br);
    p.r1x = draw_region(rng, rs);
    p.r1y = draw_region(rng, rs);
    // redraw until the second offset differs; bounded so a degenerate offset range cannot spin
    // (after kMaxRedraws the x offset is moved by one; the host restatement does the same)
    int redraws = 0;
    do {
        p.o2x = draw_offset(rng, br);
        p.o2y = draw_offset(rng, br);
        p.r2x = draw_region(rng, rs);
        p.r2y = draw_region(rng, rs);
    } while (p.o1x == p.o2x && p.o1y == p.o2y && ++redraws < kMaxRedraws);
    if (p.o1x == p.o2x && p.o1y == p.o2y) p.o2x = static_cast<int8_t>(p.o1x + 1);
    uint8_t ch1 = 0, ch2 = 0;
    if (type == kColorFeature) {
        // channel1 = feat / (numFeatures / 2.0) * 3 (double arithmetic, truncated to uint8)
        const double half = use_depth ? __ddiv_rn(static_cast<double>(F), 2.0) : __ddiv_rn(static_cast<double>(F), 1.0);
        ch1 = static_cast<uint8_t>(__dmul_rn(__ddiv_rn(static_cast<double>(feat), half), 3.0));
        ch1 %= 3;
        ch2 = static_cast<uint8_t>(__dmul_rn(__ddiv_rn(static_cast<double>(feat), __ddiv_rn(half, 3.0)), 3.0));
        ch2 %= 3;
    }
    p.ch1 = ch1;
    p.ch2 = ch2;
    p.pad = 0;
    const float scale = static_cast<float>(num_samples - 1u);
    for (int t = 0; t < T; t++) {
        const uint32_t idx = __float2uint_rz(__fmul_rn(rng.uniform(), scale));
        const Sample smp = samples[idx];
        double r = sample_response(ds, smp, p, false);
        if (isnan(r)) r = 0.0;
        raw_thr[static_cast<long long>(t) * F + feat] = __double2float_rn(r);
    }
    raw_feat[0 * F + feat] = static_cast<int8_t>(p.type);
    raw_feat[1 * F + feat] = p.o1x;
    raw_feat[2 * F + feat] = p.o1y;
    raw_feat[3 * F + feat] = p.o2x;
    raw_feat[4 * F + feat] = p.o2y;
    raw_feat[5 * F + feat] = p.r1x;
    raw_feat[6 * F + feat] = p.r1y;
    raw_feat[7 * F + feat] = p.r2x;
    raw_feat[8 * F + feat] = p.r2y;
    raw_feat[9 * F + feat] = static_cast<int8_t>(p.ch1);
    raw_feat[10 * F + feat] = static_cast<int8_t>(p.ch2);
    // getSortKey (random_tree_image.h:444-452)
    int32_t key = 0;
    key |= static_cast<uint8_t>(p.type & 0x03) << 30;
    key |= static_cast<uint8_t>(p.ch1 & 0x0F) << 26;
    key |= static_cast<uint8_t>(p.ch2 & 0x0F) << 22;
    key |= static_cast<uint8_t>((p.o1y + 127) & 0xFF) << 14;
    key |= static_cast<uint8_t>((p.o1x + 127) & 0xFF) << 6;
    keys[feat] = key;
}

// Stable rank sort of F keys: rank(i) = #{j : key_j < key_i or (key_j == key_i and j < i)};
// then scatter the feature rows and thresholds into sorted order.
__global__ void __launch_bounds__(256)
sort_features_kernel(int F, int T, const int32_t* __restrict__ keys, const int8_t* __restrict__ raw_feat,
                     const float* __restrict__ raw_thr, int8_t* __restrict__ feat, float* __restrict__ thr) {
    __shared__ int32_t s_keys[2048];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t ki = i < F ? keys[i] : 0;
    int rank = 0;
    for (int base = 0; base < F; base += 2048) {
        const int n = min(2048, F - base);
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) s_keys[j] = keys[base + j];
        __syncthreads();
        if (i < F) {
            for (int j = 0; j < n; j++) {
                const int32_t kj = s_keys[j];
                rank += (kj < ki) | ((kj == ki) & (base + j < i));
            }
        }
    }
    if (i >= F) return;
    for (int r = 0; r < 11; r++) feat[r * F + rank] = raw_feat[r * F + i];
    for (int t = 0; t < T; t++) thr[static_cast<long long>(t) * F + rank] = raw_thr[static_cast<long long>(t) * F + i];
}

}  // namespace

// One warp per feature: sorted thresholds [F][T], rank of each threshold [F][T] and the packed
// parameters. Ties keep index order, so equal thresholds get consecutive ranks.
__global__ void __launch_bounds__(256)
prepare_eval_features_kernel(int F, int T, const int8_t* __restrict__ feat, const float* __restrict__ thr,
                             FeatParams* __restrict__ packs, float* __restrict__ sorted_thr,
                             uint16_t* __restrict__ ranks) {
    const int f = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (f >= F) return;
    if (lane == 0) packs[f] = load_feature(feat, F, f);
    for (int t = lane; t < T; t += 32) {
        const float v = thr[static_cast<long long>(t) * F + f];
        int rank = 0;
        for (int j = 0; j < T; j++) {
            const float u = thr[static_cast<long long>(j) * F + f];
            rank += (u < v) | ((u == v) & (j < t));
        }
        ranks[static_cast<long long>(f) * T + t] = static_cast<uint16_t>(rank);
        sorted_thr[static_cast<long long>(f) * T + rank] = v;
    }
}

void LevelFeatures::reserve(int F_, int T_) {
    F = F_;
    T = T_;
    raw_feat.reserve(static_cast<size_t>(11) * F);
    raw_thr.reserve(static_cast<size_t>(T) * F);
    keys.reserve(F);
    feat.reserve(static_cast<size_t>(11) * F);
    thr.reserve(static_cast<size_t>(T) * F);
    packs.reserve(F);
    sorted_thr.reserve(static_cast<size_t>(T) * F);
    ranks.reserve(static_cast<size_t>(T) * F);
}

void generate_level_features(cf_context* ctx, const DsView& ds, const Sample* samples, uint32_t num_samples,
                             uint32_t seed, int box_radius, int region_size, int use_depth, LevelFeatures& lf) {
    CF_REQUIRE(num_samples > 0, "feature generation needs at least one sample");
    launch(ctx, "gen_features", dim3((lf.F + 127) / 128), dim3(128), 0, gen_features_kernel, ds, samples, num_samples,
           seed, lf.F, lf.T, box_radius, region_size, use_depth, lf.raw_feat.get(), lf.raw_thr.get(), lf.keys.get());
    launch(ctx, "sort_features", dim3((lf.F + 255) / 256), dim3(256), 0, sort_features_kernel, lf.F, lf.T,
           lf.keys.get(), lf.raw_feat.get(), lf.raw_thr.get(), lf.feat.get(), lf.thr.get());
    prepare_eval_features(ctx, lf);
}

void prepare_eval_features(cf_context* ctx, LevelFeatures& lf) {
    launch(ctx, "prepare_features", dim3((lf.F + 7) / 8), dim3(256), 0, prepare_eval_features_kernel, lf.F, lf.T,
           lf.feat.get(), lf.thr.get(), lf.packs.get(), lf.sorted_thr.get(), lf.ranks.get());
}

}  // namespace cf
