// Dense per-pixel forest prediction (kernel e).
//
// Replaces classifyKernel + normalizeProbabilitiesKernel + maxProbabilitiesKernel
// (random_tree_image_gpu.cu:1237-1453), launched once per tree per image in the reference, by one
// launch over all trees and all frames of a batch (frames may differ in size). One thread per
// pixel: its depth comes from the integral image as on the reference's CPU path
// (random_tree_image.h:140-165); each tree is walked with the exact double feature response,
// NaN going right; the leaf histograms are summed in registers, normalised by their double sum
// and arg-maxed with the lowest label winning ties (random_forest_image.cpp:307-345). The top
// levels of every tree are staged in shared memory, the rest is read through L1/L2.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "eval_fast.cuh"
#include "features.h"
#include "forest.h"

namespace cf {

namespace {

constexpr int kClassifyThreads = 256;
constexpr int kSmemNodesBudget = 2048;  // 32 KB of cached nodes per CTA
constexpr int kTreeChunk = 32;          // trees walked before their leaves are summed
constexpr int kTileW = 32, kTileH = 8;  // pixels of one classify CTA (8 warps of 8x4)

__device__ __forceinline__ float pixel_depth(const int2* D, int W, int x, int y) {
    const int2 c = __ldg(D + static_cast<long long>(y) * W + x);
    const int2 a = y > 0 ? __ldg(D + static_cast<long long>(y - 1) * W + x) : make_int2(0, 0);
    const int2 l = x > 0 ? __ldg(D + static_cast<long long>(y) * W + x - 1) : make_int2(0, 0);
    const int2 al = (x > 0 && y > 0) ? __ldg(D + static_cast<long long>(y - 1) * W + x - 1) : make_int2(0, 0);
    const int valid = c.y - (l.y + a.y - al.y);
    if (valid != 1) return 0.0f;
    const int mm = static_cast<int>(static_cast<uint32_t>(c.x) -
                                    (static_cast<uint32_t>(l.x) + static_cast<uint32_t>(a.x) - static_cast<uint32_t>(al.x)));
    if (mm <= 0) return 0.0f;
    return __fdiv_rn(static_cast<float>(mm), 1000.0f);
}

// A CTA covers 32x8 pixels, each warp an 8x4 tile, so the lanes of a warp are close in both
// directions and mostly walk the same nodes. Each lane moves on to its next tree as soon as it
// reaches a leaf (lanes do not wait at tree boundaries for the deepest path of the warp) and only
// records the leaf ([tree][threads] after the node cache); the histograms are summed afterwards,
// all lanes together, in tree order.
template <int CMAX>
__global__ void __launch_bounds__(kClassifyThreads, CMAX <= 64 ? 4 : 1)
classify_kernel(const PackedNode* __restrict__ nodes, const int* __restrict__ tree_base, int num_trees, int cache,
                const float* __restrict__ leaves, int C, const FrameDesc* __restrict__ frames, int num_frames) {
    extern __shared__ __align__(16) unsigned char smem[];
    PackedNode* s_nodes = reinterpret_cast<PackedNode*>(smem);
    uint32_t* my_leaf = reinterpret_cast<uint32_t*>(smem + sizeof(PackedNode) * num_trees * cache) + threadIdx.x;
    // which frame does this CTA serve
    int lo = 0, hi = num_frames - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (frames[mid].first_block <= static_cast<int>(blockIdx.x)) lo = mid; else hi = mid - 1;
    }
    const FrameDesc fr = frames[lo];
    // stage the top `cache` nodes of every tree
    for (int i = threadIdx.x; i < num_trees * cache; i += blockDim.x) {
        const int t = i / cache, k = i - t * cache;
        const int nt = tree_base[t + 1] - tree_base[t];
        if (k < nt) s_nodes[i] = nodes[tree_base[t] + k];
    }
    __syncthreads();
    const long long plane = static_cast<long long>(fr.width) * fr.height;
    const int b = static_cast<int>(blockIdx.x) - fr.first_block;
    const int bw = (fr.width + kTileW - 1) / kTileW;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = (b % bw) * kTileW + (warp & 3) * 8 + (lane & 7);
    const int y = (b / bw) * kTileH + (warp >> 2) * 4 + (lane >> 3);
    if (x >= fr.width || y >= fr.height) return;
    const long long p = static_cast<long long>(y) * fr.width + x;
    const float depth = pixel_depth(fr.depth, fr.width, x, y);
    EvalPixel px;
    px.color = fr.color;
    px.depth = fr.depth;
    px.x = x;
    px.y = y;
    px.d = depth;
    px.inv_d = depth > 0.0f ? __frcp_rn(depth) : 0.0f;

    float acc[CMAX];
    for (int t0 = 0; t0 < num_trees; t0 += kTreeChunk) {
        const int t1 = min(num_trees, t0 + kTreeChunk);
        int t = t0, idx = 0;
        int base = tree_base[t];
        int cached = min(cache, tree_base[t + 1] - base);
        while (t < t1) {
            const PackedNode nd = idx < cached ? s_nodes[t * cache + idx] : nodes[base + idx];
            const uint32_t meta = nd.meta;
            if (meta & 0x80000000u) {
                my_leaf[(t - t0) * kClassifyThreads] = meta & 0x7FFFFFFFu;
                if (++t < t1) {
                    base = tree_base[t];
                    cached = min(cache, tree_base[t + 1] - base);
                }
                idx = 0;
                continue;
            }
            // !(r <= threshold) for the exact double response (NaN right), decided on the fast
            // path unless the threshold lies within its error bound
            const EvalFeat ef = eval_feat_of(nd.o1x, nd.o1y, nd.o2x, nd.o2y, nd.r1x, nd.r1y, nd.r2x, nd.r2y,
                                             (meta >> 26) & 1u, (meta >> 27) & 3u, (meta >> 29) & 3u);
            idx = static_cast<int>(meta & 0x03FFFFFFu) +
                  feature_bin(px, fr.width, fr.height, ef, false, ThresholdSide{nd.threshold});
        }
        // the leaves' normalised histograms, summed in tree order as the reference sums them
        for (int tt = t0; tt < t1; tt++) {
            const float* row = leaves + static_cast<long long>(my_leaf[(tt - t0) * kClassifyThreads]) * C;
#pragma unroll
            for (int c = 0; c < CMAX; c++)
                if (c < C) acc[c] = __fadd_rn(tt == 0 ? 0.0f : acc[c], __ldg(row + c));
        }
    }
    auto acc_of = [&](int c) { return acc[c]; };
    double sum = 0.0;
#pragma unroll
    for (int c = 0; c < CMAX; c++)
        if (c < C) sum = __dadd_rn(sum, static_cast<double>(acc_of(c)));
    // RN(acc / sum) from the correctly rounded reciprocal with one correction step (Markstein,
    // IBM J. Res. Dev. 34(1), 1990): q = RN(a y), r = a - q sum exactly by FMA, RN(q + r y)
    const double inv = __drcp_rn(sum);
    float best = -1.0f;
    int label = 0;
#pragma unroll
    for (int c = 0; c < CMAX; c++) {
        if (c < C) {
            const double a = static_cast<double>(acc_of(c));
            const double q = __dmul_rn(a, inv);
            const double q1 = __fma_rn(__fma_rn(-q, sum, a), inv, q);
            const float v = __double2float_rn(q1);
            if (fr.probs) fr.probs[c * plane + p] = v;
            if (v > best) {
                best = v;
                label = c;
            }
        }
    }
    if (fr.labels) fr.labels[p] = static_cast<uint8_t>(label);
}

// ---- the plain per-image launch form (classifyImage, random_tree_image_gpu.cu:1414-1453): per image
// and tree one launch that walks that tree with the exact double response and adds the leaf
// histogram into probabilities [C][H][W] in global memory, then a normalisation launch and an
// argmax launch, each followed by a stream synchronisation as the reference's mutex-guarded loop.
__global__ void plain_classify_tree_kernel(const PackedNode* __restrict__ nodes, int base,
                                           const float* __restrict__ leaves, int C, FrameDesc fr) {
    const long long plane = static_cast<long long>(fr.width) * fr.height;
    const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= plane) return;
    const int y = static_cast<int>(p / fr.width);
    const int x = static_cast<int>(p - static_cast<long long>(y) * fr.width);
    DsView ds;
    ds.color = fr.color;
    ds.depth = fr.depth;
    ds.n = 1;
    ds.width = fr.width;
    ds.height = fr.height;
    ds.plane = plane;
    const float depth = pixel_depth(fr.depth, fr.width, x, y);
    int idx = 0;
    uint32_t meta;
    for (;;) {
        const PackedNode nd = nodes[base + idx];
        meta = nd.meta;
        if (meta & 0x80000000u) break;
        FeatParams fp;
        fp.o1x = nd.o1x;
        fp.o1y = nd.o1y;
        fp.o2x = nd.o2x;
        fp.o2y = nd.o2y;
        fp.r1x = nd.r1x;
        fp.r1y = nd.r1y;
        fp.r2x = nd.r2x;
        fp.r2y = nd.r2y;
        fp.type = static_cast<uint8_t>((meta >> 26) & 1u);
        fp.ch1 = static_cast<uint8_t>((meta >> 27) & 3u);
        fp.ch2 = static_cast<uint8_t>((meta >> 29) & 3u);
        fp.pad = 0;
        const double r = feature_response(ds, 0, x, y, depth, fp, false);
        idx = static_cast<int>(meta & 0x03FFFFFFu) + ((r <= static_cast<double>(nd.threshold)) ? 0 : 1);
    }
    const float* row = leaves + static_cast<long long>(meta & 0x7FFFFFFFu) * C;
    for (int c = 0; c < C; c++) fr.probs[c * plane + p] = __fadd_rn(fr.probs[c * plane + p], __ldg(row + c));
}

__global__ void plain_normalize_kernel(float* __restrict__ probs, int C, long long plane) {
    const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= plane) return;
    double sum = 0.0;
    for (int c = 0; c < C; c++) sum = __dadd_rn(sum, static_cast<double>(probs[c * plane + p]));
    for (int c = 0; c < C; c++)
        probs[c * plane + p] = __double2float_rn(__ddiv_rn(static_cast<double>(probs[c * plane + p]), sum));
}

__global__ void plain_argmax_kernel(const float* __restrict__ probs, int C, long long plane, uint8_t* __restrict__ labels) {
    const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= plane) return;
    float best = -1.0f;
    int label = 0;
    for (int c = 0; c < C; c++) {
        const float v = probs[c * plane + p];
        if (v > best) {
            best = v;
            label = c;
        }
    }
    labels[p] = static_cast<uint8_t>(label);
}

template <int CMAX>
void launch_classify(cf_context* ctx, cudaStream_t stream, const cf_forest* f, const FrameDesc* frames, int num_frames,
                     int blocks) {
    const size_t smem = sizeof(PackedNode) * f->num_trees * f->cache_per_tree +
                        sizeof(uint32_t) * std::min(f->num_trees, kTreeChunk) * kClassifyThreads;
    auto kernel = classify_kernel<CMAX>;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CF_CUDA_CHECK(cudaStreamIsCapturing(stream, &cs));
    if (cs == cudaStreamCaptureStatusNone)   // set before capture (an uncaptured pass runs first)
        CF_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(std::max<size_t>(smem, 1))));
    launch_on(ctx, stream, "classify", dim3(blocks), dim3(kClassifyThreads), smem, kernel, f->nodes.get(),
              f->d_tree_base.get(), f->num_trees, f->cache_per_tree, f->leaves.get(), f->C, frames, num_frames);
}

}  // namespace

int classify_blocks_for(int width, int height) {
    return ((width + kTileW - 1) / kTileW) * ((height + kTileH - 1) / kTileH);
}

void classify_frames(cf_context* ctx, const cf_forest* forest, const FrameDesc* frames_dev, int num_frames,
                     int total_blocks, cudaStream_t stream) {
    if (stream == nullptr) stream = ctx->stream;
    const int C = forest->C;
    if (C <= 8) launch_classify<8>(ctx, stream, forest, frames_dev, num_frames, total_blocks);
    else if (C <= 16) launch_classify<16>(ctx, stream, forest, frames_dev, num_frames, total_blocks);
    else if (C <= 32) launch_classify<32>(ctx, stream, forest, frames_dev, num_frames, total_blocks);
    else if (C <= 40) launch_classify<40>(ctx, stream, forest, frames_dev, num_frames, total_blocks);
    else if (C <= 64) launch_classify<64>(ctx, stream, forest, frames_dev, num_frames, total_blocks);
    else if (C <= 128) launch_classify<128>(ctx, stream, forest, frames_dev, num_frames, total_blocks);
    else launch_classify<256>(ctx, stream, forest, frames_dev, num_frames, total_blocks);
}

// detail::normalizeHistogram (random_tree.cpp:54-104)
void normalize_histogram(int C, const uint32_t* h, const uint32_t* prior, double bias, bool use_prior, double* out) {
    std::vector<double> w(C);
    double psum = 0;
    for (int i = 0; i < C; i++) psum += prior[i];
    for (int i = 0; i < C; i++) w[i] = prior[i] / psum;
    double sum = 0;
    for (int i = 0; i < C; i++) sum += h[i];
    for (int i = 0; i < C; i++) {
        out[i] = h[i] - bias * sum;
        if (out[i] < 0.0) out[i] = 0.0;
    }
    sum = 0;
    for (int i = 0; i < C; i++) sum += out[i];
    if (sum > 0)
        for (int i = 0; i < C; i++) out[i] = use_prior ? out[i] / sum * w[i] : out[i] / sum;
}

}  // namespace cf

using namespace cf;

namespace {

void predict_frames(cf_forest* f, std::vector<FrameDesc>& frames) {
    cf_context* ctx = f->ctx;
    int blocks = 0;
    for (auto& fr : frames) {
        fr.first_block = blocks;
        blocks += classify_blocks_for(fr.width, fr.height);
    }
    f->frames.reserve(frames.size());
    CF_CUDA_CHECK(cudaMemcpyAsync(f->frames.get(), frames.data(), sizeof(FrameDesc) * frames.size(),
                                  cudaMemcpyHostToDevice, ctx->stream));
    classify_frames(ctx, f, f->frames.get(), static_cast<int>(frames.size()), blocks);
}

}  // namespace

extern "C" {

cf_status cf_forest_create(cf_context* ctx, int num_trees, cf_tree* const* trees, const uint32_t* prior,
                           double histogram_bias, int use_labels_prior, cf_forest** out) {
    return guard([&] {
        CF_REQUIRE(ctx && trees && out, "cf_forest_create: NULL argument");
        CF_REQUIRE(num_trees >= 1, "cannot construct empty forest");
        make_current(ctx);
        const int C = trees[0]->C;
        for (int t = 0; t < num_trees; t++) {
            CF_REQUIRE(trees[t] != nullptr, "cf_forest_create: NULL tree");
            CF_REQUIRE(trees[t]->C == C, "different number of classes in trees");
            CF_REQUIRE(prior != nullptr || static_cast<int>(trees[t]->prior.size()) == C,
                       "cf_forest_create: no class prior given and the tree carries none");
        }
        auto* f = new cf_forest();
        std::unique_ptr<cf_forest> guard_f(f);
        f->ctx = ctx;
        f->num_trees = num_trees;
        f->C = C;
        std::vector<PackedNode> packed;
        std::vector<float> leaves;
        std::vector<int> base(num_trees + 1, 0);
        std::vector<double> norm(C);
        for (int t = 0; t < num_trees; t++) {
            const cf_tree* tr = trees[t];
            base[t] = static_cast<int>(packed.size());
            CF_REQUIRE(tr->num_nodes < (1 << 26), "tree too large for the packed node format");
            const uint32_t* pr = prior ? prior : tr->prior.data();
            for (int i = 0; i < tr->num_nodes; i++) {
                PackedNode pn;
                const int8_t* fe = &tr->feature[static_cast<size_t>(i) * 11];
                pn.o1x = fe[1];
                pn.o1y = fe[2];
                pn.o2x = fe[3];
                pn.o2y = fe[4];
                pn.r1x = fe[5];
                pn.r1y = fe[6];
                pn.r2x = fe[7];
                pn.r2y = fe[8];
                if (tr->left[i] < 0) {
                    normalize_histogram(C, &tr->hist[static_cast<size_t>(i) * C], pr, histogram_bias,
                                        use_labels_prior != 0, norm.data());
                    const int64_t row = static_cast<int64_t>(leaves.size() / C);
                    CF_REQUIRE(row < 0x7FFFFFFF, "too many leaves");
                    for (int c = 0; c < C; c++) leaves.push_back(static_cast<float>(norm[c]));
                    pn.threshold = std::nanf("");
                    pn.meta = 0x80000000u | static_cast<uint32_t>(row);
                } else {
                    CF_REQUIRE(tr->left[i] > i && tr->left[i] + 1 < tr->num_nodes, "corrupt tree: bad child index");
                    pn.threshold = tr->threshold[i];
                    pn.meta = static_cast<uint32_t>(tr->left[i]) | (static_cast<uint32_t>(fe[0] & 1) << 26) |
                              (static_cast<uint32_t>(fe[9] & 3) << 27) | (static_cast<uint32_t>(fe[10] & 3) << 29);
                }
                packed.push_back(pn);
            }
        }
        base[num_trees] = static_cast<int>(packed.size());
        f->tree_base = base;
        f->num_nodes = static_cast<int64_t>(packed.size());
        f->num_leaves = static_cast<int64_t>(leaves.size() / C);
        f->cache_per_tree = std::max(1, kSmemNodesBudget / num_trees);
        f->nodes.reserve(packed.size());
        f->d_tree_base.reserve(base.size());
        f->leaves.reserve(leaves.size());
        CF_CUDA_CHECK(cudaMemcpyAsync(f->nodes.get(), packed.data(), sizeof(PackedNode) * packed.size(),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(f->d_tree_base.get(), base.data(), sizeof(int) * base.size(),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(f->leaves.get(), leaves.data(), sizeof(float) * leaves.size(),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
        context_retain(ctx);
        *out = guard_f.release();
    });
}

cf_status cf_forest_destroy(cf_forest* forest) {
    return guard([&] {
        if (!forest) return;
        cf_context* ctx = forest->ctx;
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        delete forest;
        context_release(ctx);
    });
}

cf_status cf_forest_set_preprocessing(cf_forest* forest, int fill_depth, int cie_lab) {
    return guard([&] {
        CF_REQUIRE(forest, "cf_forest_set_preprocessing: forest is NULL");
        forest->preprocess = (fill_depth ? kPreFillDepth : 0) | (cie_lab ? kPreCieLab : 0);
    });
}

cf_status cf_forest_info(cf_forest* forest, int* num_trees, int* num_classes, int64_t* num_nodes) {
    return guard([&] {
        CF_REQUIRE(forest, "cf_forest_info: forest is NULL");
        if (num_trees) *num_trees = forest->num_trees;
        if (num_classes) *num_classes = forest->C;
        if (num_nodes) *num_nodes = forest->num_nodes;
    });
}

cf_status cf_predict_dataset(cf_forest* forest, cf_dataset* ds, int first, int count, float* probabilities,
                             uint8_t* labels) {
    return guard([&] {
        CF_REQUIRE(forest && ds, "cf_predict_dataset: NULL argument");
        CF_REQUIRE(first >= 0 && count >= 1 && first + count <= ds->n, "cf_predict_dataset: image range");
        CF_REQUIRE(ds->ctx == forest->ctx, "cf_predict_dataset: dataset and forest belong to different contexts");
        make_current(forest->ctx);
        const long long plane = static_cast<long long>(ds->width) * ds->height;
        std::vector<FrameDesc>& frames = forest->h_frames;
        frames.resize(count);
        for (int i = 0; i < count; i++) {
            FrameDesc& fr = frames[i];
            fr.color = ds->color.get() + (first + i) * plane * 3;
            fr.depth = ds->depth.get() + (first + i) * plane;
            fr.probs = probabilities ? probabilities + static_cast<long long>(i) * forest->C * plane : nullptr;
            fr.labels = labels ? labels + static_cast<long long>(i) * plane : nullptr;
            fr.width = ds->width;
            fr.height = ds->height;
            fr.pad = 0;
        }
        predict_frames(forest, frames);
    });
}

cf_status cf_predict_host(cf_forest* forest, int count, int width, int height, const uint8_t* rgb,
                          const uint16_t* depth_mm, float* probabilities, uint8_t* labels) {
    return guard([&] {
        CF_REQUIRE(forest && rgb && depth_mm, "cf_predict_host: NULL argument");
        CF_REQUIRE(count >= 1 && width >= 1 && height >= 1, "cf_predict_host: empty input");
        cf_context* ctx = forest->ctx;
        make_current(ctx);
        const size_t plane = static_cast<size_t>(width) * height;
        forest->raw_rgb.reserve(plane * 3 * count);
        forest->raw_depth.reserve(plane * count);
        forest->color.reserve(plane * 3 * count);
        forest->depth.reserve(plane * count);
        if (probabilities) forest->probs.reserve(plane * forest->C * count);
        forest->labels.reserve(plane * count);
        CF_CUDA_CHECK(cudaMemcpyAsync(forest->raw_rgb.get(), rgb, plane * 3 * count, cudaMemcpyHostToDevice, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(forest->raw_depth.get(), depth_mm, plane * 2 * count, cudaMemcpyHostToDevice,
                                      ctx->stream));
        integrate_frames(ctx, forest->raw_rgb.get(), forest->raw_depth.get(), count, width, height, forest->color.get(),
                         forest->depth.get(), ctx->stream, forest->preprocess);
        std::vector<FrameDesc>& frames = forest->h_frames;
        frames.resize(count);
        for (int i = 0; i < count; i++) {
            FrameDesc& fr = frames[i];
            fr.color = forest->color.get() + plane * 3 * i;
            fr.depth = forest->depth.get() + plane * i;
            fr.probs = probabilities ? forest->probs.get() + plane * forest->C * i : nullptr;
            fr.labels = forest->labels.get() + plane * i;
            fr.width = width;
            fr.height = height;
            fr.pad = 0;
        }
        predict_frames(forest, frames);
        if (probabilities)
            CF_CUDA_CHECK(cudaMemcpyAsync(probabilities, forest->probs.get(), sizeof(float) * plane * forest->C * count,
                                          cudaMemcpyDeviceToHost, ctx->stream));
        if (labels)
            CF_CUDA_CHECK(cudaMemcpyAsync(labels, forest->labels.get(), plane * count, cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_predict_dataset_host(cf_forest* forest, cf_dataset* ds, int first, int count, float* probabilities,
                                  uint8_t* labels) {
    return guard([&] {
        CF_REQUIRE(forest && ds, "cf_predict_dataset_host: NULL argument");
        CF_REQUIRE(first >= 0 && count >= 1 && first + count <= ds->n, "cf_predict_dataset_host: image range");
        CF_REQUIRE(ds->ctx == forest->ctx, "cf_predict_dataset_host: dataset and forest belong to different contexts");
        cf_context* ctx = forest->ctx;
        make_current(ctx);
        const size_t plane = static_cast<size_t>(ds->width) * ds->height;
        if (probabilities) forest->probs.reserve(plane * forest->C * count);
        forest->labels.reserve(plane * count);
        std::vector<FrameDesc>& frames = forest->h_frames;
        frames.resize(count);
        for (int i = 0; i < count; i++) {
            FrameDesc& fr = frames[i];
            fr.color = ds->color.get() + (first + i) * plane * 3;
            fr.depth = ds->depth.get() + (first + i) * plane;
            fr.probs = probabilities ? forest->probs.get() + plane * forest->C * i : nullptr;
            fr.labels = forest->labels.get() + plane * i;
            fr.width = ds->width;
            fr.height = ds->height;
            fr.pad = 0;
        }
        predict_frames(forest, frames);
        if (probabilities)
            CF_CUDA_CHECK(cudaMemcpyAsync(probabilities, forest->probs.get(), sizeof(float) * plane * forest->C * count,
                                          cudaMemcpyDeviceToHost, ctx->stream));
        if (labels)
            CF_CUDA_CHECK(cudaMemcpyAsync(labels, forest->labels.get(), plane * count, cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_normalize_histogram(int num_classes, const uint32_t* histogram, const uint32_t* prior,
                                 double histogram_bias, int use_labels_prior, double* out) {
    return guard([&] {
        CF_REQUIRE(histogram && prior && out, "cf_normalize_histogram: NULL argument");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_normalize_histogram: classes must be in [1, 256]");
        uint64_t psum = 0;
        for (int c = 0; c < num_classes; c++) psum += prior[c];
        CF_REQUIRE(psum > 0, "cf_normalize_histogram: empty class prior");
        normalize_histogram(num_classes, histogram, prior, histogram_bias, use_labels_prior != 0, out);
    });
}

cf_status cf_predict_dataset_plain(cf_forest* forest, cf_dataset* ds, int first, int count, float* probabilities,
                                   uint8_t* labels) {
    return guard([&] {
        CF_REQUIRE(forest && ds, "cf_predict_dataset_plain: NULL argument");
        CF_REQUIRE(first >= 0 && count >= 1 && first + count <= ds->n, "cf_predict_dataset_plain: image range");
        CF_REQUIRE(ds->ctx == forest->ctx, "cf_predict_dataset_plain: dataset and forest belong to different contexts");
        cf_context* ctx = forest->ctx;
        make_current(ctx);
        const int C = forest->C;
        const long long plane = static_cast<long long>(ds->width) * ds->height;
        const unsigned blocks = static_cast<unsigned>((plane + 255) / 256);
        if (!probabilities) forest->probs.reserve(static_cast<size_t>(plane) * C);
        if (!labels) forest->labels.reserve(static_cast<size_t>(plane));
        cudaStream_t st = ctx->stream;
        for (int i = 0; i < count; i++) {
            FrameDesc fr;
            fr.color = ds->color.get() + (first + i) * plane * 3;
            fr.depth = ds->depth.get() + (first + i) * plane;
            fr.probs = probabilities ? probabilities + static_cast<long long>(i) * C * plane : forest->probs.get();
            fr.labels = labels ? labels + static_cast<long long>(i) * plane : forest->labels.get();
            fr.width = ds->width;
            fr.height = ds->height;
            fr.first_block = 0;
            fr.pad = 0;
            CF_CUDA_CHECK(cudaMemsetAsync(fr.probs, 0, sizeof(float) * C * plane, st));
            for (int t = 0; t < forest->num_trees; t++) {
                launch(ctx, "plain_classify", dim3(blocks), dim3(256), 0, plain_classify_tree_kernel, forest->nodes.get(),
                       forest->tree_base[t], forest->leaves.get(), C, fr);
                CF_CUDA_CHECK(cudaStreamSynchronize(st));
            }
            launch(ctx, "plain_normalize", dim3(blocks), dim3(256), 0, plain_normalize_kernel, fr.probs, C, plane);
            CF_CUDA_CHECK(cudaStreamSynchronize(st));
            launch(ctx, "plain_argmax", dim3(blocks), dim3(256), 0, plain_argmax_kernel, fr.probs, C, plane, fr.labels);
            CF_CUDA_CHECK(cudaStreamSynchronize(st));
        }
    });
}

cf_status cf_predict_host_plain(cf_forest* forest, int count, int width, int height, const uint8_t* rgb,
                                const uint16_t* depth_mm, float* probabilities, uint8_t* labels) {
    return guard([&] {
        CF_REQUIRE(forest && rgb && depth_mm, "cf_predict_host_plain: NULL argument");
        CF_REQUIRE(count >= 1 && width >= 1 && height >= 1, "cf_predict_host_plain: empty input");
        cf_context* ctx = forest->ctx;
        make_current(ctx);
        const int C = forest->C;
        const size_t plane = static_cast<size_t>(width) * height;
        const unsigned blocks = static_cast<unsigned>((plane + 255) / 256);
        forest->raw_rgb.reserve(plane * 3);
        forest->raw_depth.reserve(plane);
        forest->color.reserve(plane * 3);
        forest->depth.reserve(plane);
        forest->probs.reserve(plane * C);
        forest->labels.reserve(plane);
        // the reference copies the probabilities back for every image, requested or not
        std::vector<float> host_probs(probabilities ? 0 : plane * C);
        std::vector<uint8_t> host_labels(labels ? 0 : plane);
        cudaStream_t st = ctx->stream;
        for (int i = 0; i < count; i++) {
            CF_CUDA_CHECK(cudaMemcpyAsync(forest->raw_rgb.get(), rgb + plane * 3 * i, plane * 3, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(forest->raw_depth.get(), depth_mm + plane * i, plane * 2, cudaMemcpyHostToDevice,
                                          st));
            integrate_frames(ctx, forest->raw_rgb.get(), forest->raw_depth.get(), 1, width, height, forest->color.get(),
                             forest->depth.get(), ctx->stream, forest->preprocess);
            FrameDesc fr;
            fr.color = forest->color.get();
            fr.depth = forest->depth.get();
            fr.probs = forest->probs.get();
            fr.labels = forest->labels.get();
            fr.width = width;
            fr.height = height;
            fr.first_block = 0;
            fr.pad = 0;
            CF_CUDA_CHECK(cudaMemsetAsync(fr.probs, 0, sizeof(float) * C * plane, st));
            for (int t = 0; t < forest->num_trees; t++) {
                launch(ctx, "plain_classify", dim3(blocks), dim3(256), 0, plain_classify_tree_kernel, forest->nodes.get(),
                       forest->tree_base[t], forest->leaves.get(), C, fr);
                CF_CUDA_CHECK(cudaStreamSynchronize(st));
            }
            const long long pl = static_cast<long long>(plane);
            launch(ctx, "plain_normalize", dim3(blocks), dim3(256), 0, plain_normalize_kernel, fr.probs, C, pl);
            CF_CUDA_CHECK(cudaStreamSynchronize(st));
            launch(ctx, "plain_argmax", dim3(blocks), dim3(256), 0, plain_argmax_kernel, fr.probs, C, pl, fr.labels);
            CF_CUDA_CHECK(cudaStreamSynchronize(st));
            float* pd = probabilities ? probabilities + plane * C * i : host_probs.data();
            uint8_t* ld = labels ? labels + plane * i : host_labels.data();
            CF_CUDA_CHECK(cudaMemcpyAsync(pd, fr.probs, sizeof(float) * plane * C, cudaMemcpyDeviceToHost, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(ld, fr.labels, plane, cudaMemcpyDeviceToHost, st));
            CF_CUDA_CHECK(cudaStreamSynchronize(st));
        }
    });
}

}  // extern "C"

// ---- batch prediction captured as a CUDA graph ----------------------------------------------------
struct cf_predict_graph {
    cf_forest* forest = nullptr;
    int count = 0, width = 0, height = 0;
    bool with_probs = false;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;   // kernel nodes per replay
    cf::PinnedBuffer h_rgb, h_depth, h_probs, h_labels;
    cf::DevArray<uint8_t> rgb;
    cf::DevArray<uint16_t> depth_mm;
    cf::DevArray<float> color;
    cf::DevArray<int2> dint;
    cf::DevArray<float> probs;
    cf::DevArray<uint8_t> labels;
    cf::DevArray<cf::FrameDesc> frames;

    ~cf_predict_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// One batch: pinned inputs -> device, integral images, classification, results -> pinned outputs.
void enqueue_graph_batch(cf_predict_graph* g, int blocks) {
    cf_context* ctx = g->forest->ctx;
    const size_t plane = static_cast<size_t>(g->width) * g->height;
    const size_t n = static_cast<size_t>(g->count);
    CF_CUDA_CHECK(cudaMemcpyAsync(g->rgb.get(), g->h_rgb.get(), plane * 3 * n, cudaMemcpyHostToDevice, g->stream));
    CF_CUDA_CHECK(cudaMemcpyAsync(g->depth_mm.get(), g->h_depth.get(), plane * 2 * n, cudaMemcpyHostToDevice, g->stream));
    integrate_frames(ctx, g->rgb.get(), g->depth_mm.get(), g->count, g->width, g->height, g->color.get(), g->dint.get(),
                     g->stream, g->forest->preprocess);
    classify_frames(ctx, g->forest, g->frames.get(), g->count, blocks, g->stream);
    CF_CUDA_CHECK(cudaMemcpyAsync(g->h_labels.get(), g->labels.get(), plane * n, cudaMemcpyDeviceToHost, g->stream));
    if (g->with_probs)
        CF_CUDA_CHECK(cudaMemcpyAsync(g->h_probs.get(), g->probs.get(), sizeof(float) * plane * g->forest->C * n,
                                      cudaMemcpyDeviceToHost, g->stream));
}

}  // namespace

extern "C" {

cf_status cf_predict_graph_create(cf_forest* forest, int count, int width, int height, int with_probabilities,
                                  cf_predict_graph** out) {
    return guard([&] {
        CF_REQUIRE(forest && out, "cf_predict_graph_create: NULL argument");
        CF_REQUIRE(count >= 1 && width >= 1 && height >= 1, "cf_predict_graph_create: empty batch");
        cf_context* ctx = forest->ctx;
        make_current(ctx);
        auto* g = new cf_predict_graph();
        std::unique_ptr<cf_predict_graph> own(g);
        g->forest = forest;
        g->count = count;
        g->width = width;
        g->height = height;
        g->with_probs = with_probabilities != 0;
        const size_t plane = static_cast<size_t>(width) * height;
        const size_t n = static_cast<size_t>(count);
        const int C = forest->C;
        g->h_rgb.reserve(plane * 3 * n);
        g->h_depth.reserve(plane * 2 * n);
        g->h_labels.reserve(plane * n);
        if (g->with_probs) g->h_probs.reserve(sizeof(float) * plane * C * n);
        std::memset(g->h_rgb.get(), 0, plane * 3 * n);
        std::memset(g->h_depth.get(), 0, plane * 2 * n);
        g->rgb.reserve(plane * 3 * n);
        g->depth_mm.reserve(plane * n);
        g->color.reserve(plane * 3 * n);
        g->dint.reserve(plane * n);
        g->labels.reserve(plane * n);
        if (g->with_probs) g->probs.reserve(plane * C * n);
        std::vector<FrameDesc> frames(n);
        int blocks = 0;
        for (size_t i = 0; i < n; i++) {
            FrameDesc& fr = frames[i];
            fr.color = g->color.get() + plane * 3 * i;
            fr.depth = g->dint.get() + plane * i;
            fr.probs = g->with_probs ? g->probs.get() + plane * C * i : nullptr;
            fr.labels = g->labels.get() + plane * i;
            fr.width = width;
            fr.height = height;
            fr.first_block = blocks;
            fr.pad = 0;
            blocks += classify_blocks_for(width, height);
        }
        g->frames.reserve(n);
        CF_CUDA_CHECK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        CF_CUDA_CHECK(cudaMemcpyAsync(g->frames.get(), frames.data(), sizeof(FrameDesc) * n, cudaMemcpyHostToDevice,
                                      g->stream));
        // one uncaptured pass sets the kernels' attributes and checks the pipeline, then capture
        enqueue_graph_batch(g, blocks);
        CF_CUDA_CHECK(cudaStreamSynchronize(g->stream));
        const int64_t before = ctx->launches.load();
        CF_CUDA_CHECK(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_graph_batch(g, blocks);
        } catch (...) {
            cudaGraph_t broken = nullptr;
            cudaStreamEndCapture(g->stream, &broken);
            if (broken) cudaGraphDestroy(broken);
            throw;
        }
        CF_CUDA_CHECK(cudaStreamEndCapture(g->stream, &g->graph));
        g->kernels = ctx->launches.load() - before;
        ctx->launches -= g->kernels;   // counted when the graph runs
        CF_CUDA_CHECK(cudaGraphInstantiate(&g->exec, g->graph, 0));
        context_retain(ctx);
        *out = own.release();
    });
}

cf_status cf_predict_graph_buffers(cf_predict_graph* g, uint8_t** rgb, uint16_t** depth_mm, float** probabilities,
                                   uint8_t** labels) {
    return guard([&] {
        CF_REQUIRE(g, "cf_predict_graph_buffers: graph is NULL");
        if (rgb) *rgb = static_cast<uint8_t*>(g->h_rgb.get());
        if (depth_mm) *depth_mm = static_cast<uint16_t*>(g->h_depth.get());
        if (probabilities) *probabilities = g->with_probs ? static_cast<float*>(g->h_probs.get()) : nullptr;
        if (labels) *labels = static_cast<uint8_t*>(g->h_labels.get());
    });
}

cf_status cf_predict_graph_run(cf_predict_graph* g) {
    return guard([&] {
        CF_REQUIRE(g, "cf_predict_graph_run: graph is NULL");
        cf_context* ctx = g->forest->ctx;
        make_current(ctx);
        CF_CUDA_CHECK(cudaGraphLaunch(g->exec, g->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(g->stream));
        ctx->launches += g->kernels;
    });
}

cf_status cf_predict_graph_destroy(cf_predict_graph* g) {
    return guard([&] {
        if (!g) return;
        cf_context* ctx = g->forest->ctx;
        cudaSetDevice(ctx->device);
        if (g->stream) cudaStreamSynchronize(g->stream);
        delete g;
        context_release(ctx);
    });
}

}  // extern "C"
