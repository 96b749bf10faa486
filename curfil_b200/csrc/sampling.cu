// Device class-uniform sampling of a tree's training pixels (project extension).
//
// The reference draws classUniform samples with one reservoir per class over every pixel of the
// tree's images (random_tree_image.cpp:919-1014); with several threads it merges per-thread
// reservoirs in completion order, so its samples are not reproducible. This sampler defines the
// draw deterministically and in parallel:
//   - every eligible pixel (label not ignored, depth > 0) of image list position k, pixel p gets the
//     key Philox4x32-10(key = (randomSeed, 0x53414D50), counter = (k * H * W + p, 0, 0, 0))[0],
//     randomSeed being the draw the reference takes from the tree's RandomSource for the sampler;
//   - each class keeps its `per_class` eligible pixels with the smallest (key, k * H * W + p): a
//     uniformly random subset, as a reservoir yields;
//   - the samples are ordered by (k, label, y / 10, x / 10, y, x), the reference's block-sort key
//     (random_tree_image.cpp:776-802) completed to a total order.
// The GPU counts eligible pixels per class (and the class prior), then keeps only pixels whose key
// lies below a per-class cut chosen so that at least `per_class` of them survive with overwhelming
// probability (the cut is raised and the pass repeated otherwise); the host orders the survivors.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "sampling.h"

namespace cf {

namespace {

constexpr uint32_t kSampleKey1 = 0x53414D50u;

__device__ __forceinline__ uint32_t philox_first(uint32_t k0, uint32_t k1, uint32_t ctr) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t c0 = ctr, c1 = 0, c2 = 0, c3 = 0;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        const uint32_t hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
        const uint32_t hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    return c0;
}

// class prior over all pixels and eligible pixels per class, of the listed images
__global__ void tree_pixel_counts_kernel(const uint8_t* __restrict__ labels, const uint16_t* __restrict__ depth,
                                         const int* __restrict__ images, long long plane, long long total, int C,
                                         const uint8_t* __restrict__ ignored, uint32_t* prior, uint32_t* eligible,
                                         int* bad_label) {
    __shared__ uint32_t s_prior[256], s_elig[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s_prior[i] = s_elig[i] = 0u;
    __syncthreads();
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long k = i / plane, p = i - k * plane;
        const long long src = static_cast<long long>(images[k]) * plane + p;
        const int label = labels[src];
        if (label >= C) {
            *bad_label = 1;
            continue;
        }
        atomicAdd(&s_prior[label], 1u);
        if (!ignored[label] && depth[src] > 0) atomicAdd(&s_elig[label], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < C; i += blockDim.x) {
        if (s_prior[i]) atomicAdd(&prior[i], s_prior[i]);
        if (s_elig[i]) atomicAdd(&eligible[i], s_elig[i]);
    }
}

struct Candidate {
    uint32_t key;
    uint32_t idx;    // k * plane + p
    uint32_t label;
    uint32_t pad;
};

// eligible pixels whose key lies below their class's cut, appended in any order
__global__ void tree_pixel_candidates_kernel(const uint8_t* __restrict__ labels, const uint16_t* __restrict__ depth,
                                             const int* __restrict__ images, long long plane, long long total,
                                             const uint8_t* __restrict__ ignored,
                                             const unsigned long long* __restrict__ cut, uint32_t k0,
                                             Candidate* out, unsigned long long capacity,
                                             unsigned long long* count) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long k = i / plane, p = i - k * plane;
        const long long src = static_cast<long long>(images[k]) * plane + p;
        const int label = labels[src];
        if (ignored[label] || depth[src] == 0) continue;
        const uint32_t key = philox_first(k0, kSampleKey1, static_cast<uint32_t>(i));
        if (static_cast<unsigned long long>(key) >= cut[label]) continue;
        const unsigned long long pos = atomicAdd(count, 1ull);
        if (pos < capacity) out[pos] = Candidate{key, static_cast<uint32_t>(i), static_cast<uint32_t>(label), 0u};
    }
}

}  // namespace

void DeviceFrames::upload(cf_context* ctx, int num_images, int width, int height, const uint8_t* labels_host,
                          const uint16_t* depth_host) {
    n = num_images;
    W = width;
    H = height;
    if (!stream) CF_CUDA_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    const size_t px = static_cast<size_t>(n) * W * H;
    labels.reserve(px);
    depth.reserve(px);
    images.reserve(n);
    ignored.reserve(256);
    counts.reserve(512);
    bad.reserve(1);
    cut.reserve(256);
    count.reserve(1);
    CF_CUDA_CHECK(cudaMemcpyAsync(labels.get(), labels_host, px, cudaMemcpyHostToDevice, stream));
    CF_CUDA_CHECK(cudaMemcpyAsync(depth.get(), depth_host, px * 2, cudaMemcpyHostToDevice, stream));
    CF_CUDA_CHECK(cudaStreamSynchronize(stream));
    (void)ctx;
}

std::vector<cf_sample> sample_class_uniform_device(cf_context* ctx, DeviceFrames& fr,
                                                   const std::vector<int>& images, const uint16_t* depth_host,
                                                   int C, const uint8_t* ignored_host, int subsample_count,
                                                   RandomSource& rs, uint8_t flip, std::vector<uint32_t>* prior) {
    const long long plane = static_cast<long long>(fr.W) * fr.H;
    const long long total = plane * static_cast<long long>(images.size());
    CF_REQUIRE(total < (1LL << 32), "device sampling: the tree's images hold more than 2^32 pixels");
    int numLabels = C;
    std::vector<uint8_t> ign(256, 0);
    for (int c = 0; c < C; c++)
        if (ignored_host && ignored_host[c]) {
            ign[c] = 1;
            numLabels--;
        }
    CF_REQUIRE(numLabels > 0, "no classes left to sample");
    const size_t per_class = static_cast<size_t>(
        std::ceil(images.size() * static_cast<double>(subsample_count) / static_cast<double>(numLabels)));
    // the draws the reference takes for its sampler (randomSeed) and its merge sampler
    const uint32_t k0 = static_cast<uint32_t>(rs.uniform(0xFFFFFF).next());
    (void)rs.uniform(0x7FFFFFFF);

    cudaStream_t st = fr.stream;
    CF_REQUIRE(st != nullptr && images.size() <= static_cast<size_t>(fr.n), "device sampling: frames not uploaded");
    CF_CUDA_CHECK(cudaMemcpyAsync(fr.images.get(), images.data(), sizeof(int) * images.size(), cudaMemcpyHostToDevice, st));
    CF_CUDA_CHECK(cudaMemcpyAsync(fr.ignored.get(), ign.data(), 256, cudaMemcpyHostToDevice, st));
    CF_CUDA_CHECK(cudaMemsetAsync(fr.counts.get(), 0, sizeof(uint32_t) * 2 * C, st));
    CF_CUDA_CHECK(cudaMemsetAsync(fr.bad.get(), 0, sizeof(int), st));
    const int grid = ctx->num_sms * 8;
    launch_on(ctx, st, "sample_counts", dim3(grid), dim3(256), 0, tree_pixel_counts_kernel, fr.labels.get(),
              fr.depth.get(), fr.images.get(), plane, total, C, fr.ignored.get(), fr.counts.get(), fr.counts.get() + C,
              fr.bad.get());
    std::vector<uint32_t> counts(2 * C);
    int bad = 0;
    CF_CUDA_CHECK(cudaMemcpyAsync(counts.data(), fr.counts.get(), sizeof(uint32_t) * 2 * C, cudaMemcpyDeviceToHost, st));
    CF_CUDA_CHECK(cudaMemcpyAsync(&bad, fr.bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    CF_CUDA_CHECK(cudaStreamSynchronize(st));
    CF_REQUIRE(!bad, "label image holds a label >= number of classes");
    if (prior) prior->assign(counts.begin(), counts.begin() + C);
    for (int c = 0; c < C; c++)
        if (!ign[c]) CF_REQUIRE(counts[C + c] >= per_class, "failed to sample enough pixels");

    // keys are uniform on [0, 2^32): a cut at (m + 8 sqrt(m) + 32) / eligible keeps >= m per class
    // unless the count deviates by more than 8 standard deviations; the margin grows on a retry
    static_assert(sizeof(Candidate) == sizeof(uint4), "candidate record is 16 bytes");
    std::vector<std::vector<Candidate>> by_class(C);
    for (double margin = 8.0;; margin *= 4.0) {
        std::vector<unsigned long long> cut(256, 0ull);
        double expected = 0;
        for (int c = 0; c < C; c++) {
            if (ign[c]) continue;
            const double m = static_cast<double>(per_class);
            const double frac = std::min(1.0, (m + margin * std::sqrt(m) + 32.0) / counts[C + c]);
            cut[c] = frac >= 1.0 ? (1ull << 32) : static_cast<unsigned long long>(std::ceil(frac * 4294967296.0));
            expected += frac * counts[C + c];
        }
        const unsigned long long capacity = static_cast<unsigned long long>(expected * 1.05) + 4096;
        if (fr.candidates.capacity() < capacity) {
            CF_CUDA_CHECK(cudaStreamSynchronize(st));
            fr.candidates.reserve(capacity);
        }
        Candidate* d_cand = reinterpret_cast<Candidate*>(fr.candidates.get());
        CF_CUDA_CHECK(cudaMemcpyAsync(fr.cut.get(), cut.data(), sizeof(unsigned long long) * 256, cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemsetAsync(fr.count.get(), 0, sizeof(unsigned long long), st));
        launch_on(ctx, st, "sample_candidates", dim3(grid), dim3(256), 0, tree_pixel_candidates_kernel, fr.labels.get(),
                  fr.depth.get(), fr.images.get(), plane, total, fr.ignored.get(), fr.cut.get(), k0, d_cand, capacity,
                  fr.count.get());
        unsigned long long n = 0;
        CF_CUDA_CHECK(cudaMemcpyAsync(&n, fr.count.get(), sizeof(n), cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        if (n > capacity) continue;   // more survivors than room: retry with a larger buffer
        std::vector<Candidate> cand(n);
        CF_CUDA_CHECK(cudaMemcpyAsync(cand.data(), d_cand, sizeof(Candidate) * n, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        for (auto& v : by_class) v.clear();
        for (const Candidate& x : cand) by_class[x.label].push_back(x);
        bool enough = true;
        for (int c = 0; c < C; c++)
            if (!ign[c] && by_class[c].size() < per_class) enough = false;
        if (enough) break;
    }
    // per class the quota of smallest (key, idx); then the order (k, label, y/10, x/10, y, x) as one
    // 64-bit key: k < 2^16 images, label < 2^8, y/10 and x/10 < 2^12, y%10 and x%10 < 2^4
    CF_REQUIRE(images.size() < (1u << 16) && fr.W <= 40950 && fr.H <= 40950, "device sampling: frames too large");
    std::vector<std::pair<uint64_t, uint32_t>> order;   // (order key, k * plane + p)
    order.reserve(per_class * numLabels);
    for (int c = 0; c < C; c++) {
        if (ign[c]) continue;
        auto& v = by_class[c];
        auto less = [](const Candidate& a, const Candidate& b) { return a.key != b.key ? a.key < b.key : a.idx < b.idx; };
        std::nth_element(v.begin(), v.begin() + (per_class - 1), v.end(), less);
        for (size_t j = 0; j < per_class; j++) {
            const uint64_t k = v[j].idx / plane, p = v[j].idx - k * plane;
            const uint64_t y = p / fr.W, x = p % fr.W;
            const uint64_t key = (k << 48) | (static_cast<uint64_t>(c) << 40) | ((y / 10) << 28) | ((x / 10) << 16) |
                                 ((y % 10) << 4) | (x % 10);
            order.emplace_back(key, v[j].idx);
        }
    }
    std::sort(order.begin(), order.end());
    std::vector<cf_sample> out(order.size());
    for (size_t j = 0; j < order.size(); j++) {
        const long long idx = order[j].second;
        const long long k = idx / plane, p = idx - k * plane;
        const uint16_t mm = depth_host[static_cast<long long>(images[k]) * plane + p];
        cf_sample& s = out[j];
        s.x = static_cast<uint16_t>(p % fr.W);
        s.y = static_cast<uint16_t>(p / fr.W);
        s.image = static_cast<uint32_t>(k);
        s.depth = static_cast<float>(static_cast<int>(mm)) / 1000.0f;
        s.label = static_cast<uint8_t>((order[j].first >> 40) & 0xFF);
        s.flip = flip;
        s.reserved = 0;
    }
    return out;
}

}  // namespace cf
