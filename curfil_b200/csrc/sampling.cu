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
// All on the GPU: the eligible pixels are counted per class (with the class prior); only pixels whose
// key lies below a per-class cut, chosen so that at least `per_class` of them survive with
// overwhelming probability, become candidates (the cut is raised and the pass repeated otherwise);
// radix sorts order the candidates by (class, key, pixel), the first `per_class` of every class are
// taken, and a last sort puts the samples in the block order. Only the samples go back to the host.
// The radix sorts are CUB's (cub::DeviceRadixSort, stable), as the reference sorts with Thrust.
#include <algorithm>
#include <cmath>
#include <cstring>

#include <cub/device/device_radix_sort.cuh>

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

// candidates -> (pixel index, (class << 32) | key) pairs, for the first sort (by pixel index)
__global__ void candidate_pairs_kernel(const uint4* __restrict__ cand, unsigned long long n, uint32_t* __restrict__ idx,
                                       unsigned long long* __restrict__ class_key, uint32_t* __restrict__ class_count) {
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const uint4 c = cand[i];   // {key, idx, label, pad}
        idx[i] = c.y;
        class_key[i] = (static_cast<unsigned long long>(c.z) << 32) | c.x;
        atomicAdd(&class_count[c.z], 1u);
    }
}

// the first per_class candidates of every sampled class (candidates sorted by (class, key, pixel)),
// with their block-order key (k, label, y/10, x/10, y%10, x%10)
__global__ void select_kernel(const uint32_t* __restrict__ sorted_idx, const uint32_t* __restrict__ class_start,
                              const uint8_t* __restrict__ classes, int n_classes, unsigned long long per_class,
                              long long plane, int W, unsigned long long* __restrict__ order_key,
                              uint32_t* __restrict__ order_idx) {
    const unsigned long long total = per_class * static_cast<unsigned long long>(n_classes);
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const int ci = static_cast<int>(i / per_class);
        const unsigned long long j = i - static_cast<unsigned long long>(ci) * per_class;
        const int c = classes[ci];
        const uint32_t idx = sorted_idx[class_start[c] + j];
        const unsigned long long k = idx / static_cast<unsigned long long>(plane);
        const unsigned long long p = idx - k * static_cast<unsigned long long>(plane);
        const unsigned long long y = p / W, x = p % W;
        order_key[i] = (k << 48) | (static_cast<unsigned long long>(c) << 40) | ((y / 10) << 28) | ((x / 10) << 16) |
                       ((y % 10) << 4) | (x % 10);
        order_idx[i] = idx;
    }
}

// the ordered samples: pixel, image position, depth in metres from the millimetre frame, label, flip
__global__ void emit_samples_kernel(const unsigned long long* __restrict__ order_key, const uint32_t* __restrict__ idx,
                                    unsigned long long n, const int* __restrict__ images,
                                    const uint16_t* __restrict__ depth, long long plane, int W, uint8_t flip,
                                    cf_sample* __restrict__ out) {
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const unsigned long long k = idx[i] / static_cast<unsigned long long>(plane);
        const unsigned long long p = idx[i] - k * static_cast<unsigned long long>(plane);
        const uint16_t mm = depth[static_cast<long long>(images[k]) * plane + static_cast<long long>(p)];
        cf_sample s;
        s.x = static_cast<uint16_t>(p % W);
        s.y = static_cast<uint16_t>(p / W);
        s.image = static_cast<uint32_t>(k);
        s.depth = __fdiv_rn(static_cast<float>(static_cast<int>(mm)), 1000.0f);
        s.label = static_cast<uint8_t>((order_key[i] >> 40) & 0xFF);
        s.flip = flip;
        s.reserved = 0;
        out[i] = s;
    }
}

// ---- pixelUniform (random_tree_image.cpp:840-883) -----------------------------------------------
// Every sample draws its pixel from two fresh Samplers (mt19937 seeded with consecutive seeds of the
// tree's RandomSource, Boost uniform_int on [0, W-1] and [0, H-1]) until the label is not ignored.
// Samplers of different samples are independent, so every sample is one thread. The first 227 outputs
// of an mt19937 depend only on its initial state words i, i + 1 and i + 397 (the first twist of word
// i reads no word it has already changed), so they are produced without the 624-word state; a sample
// that needs more draws (the ignored classes would have to cover almost every pixel) walks the full
// state in local memory.
struct MtHead {
    // init recurrence x[i] = 1812433253 * (x[i-1] ^ (x[i-1] >> 30)) + i at two cursors: i and i + 397
    uint32_t a, a_next, c;
    uint32_t i;
    __device__ explicit MtHead(uint32_t seed) : a(seed), i(0) {
        uint32_t x = seed;
        for (uint32_t k = 1; k <= 397; k++) {
            x = 1812433253u * (x ^ (x >> 30)) + k;
            if (k == 1) a_next = x;
        }
        c = x;
    }
    __device__ static uint32_t temper(uint32_t y) {
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }
    // output i, for i < 227
    __device__ uint32_t next() {
        const uint32_t y = (a & 0x80000000u) | (a_next & 0x7fffffffu);
        const uint32_t v = c ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        i++;
        a = a_next;
        a_next = 1812433253u * (a_next ^ (a_next >> 30)) + (i + 1);
        c = 1812433253u * (c ^ (c >> 30)) + (i + 397);
        return temper(v);
    }
};

// the full generator for a sample that needs more than 226 draws from one Sampler
struct MtFull {
    uint32_t mt[624];
    int idx;
    __device__ explicit MtFull(uint32_t seed) : idx(624) {
        mt[0] = seed;
        for (int k = 1; k < 624; k++) mt[k] = 1812433253u * (mt[k - 1] ^ (mt[k - 1] >> 30)) + k;
    }
    __device__ uint32_t next() {
        if (idx >= 624) {
            for (int k = 0; k < 624; k++) {
                const uint32_t y = (mt[k] & 0x80000000u) | (mt[(k + 1) % 624] & 0x7fffffffu);
                mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
            }
            idx = 0;
        }
        return MtHead::temper(mt[idx++]);
    }
};

// Boost uniform_int on [0, range] over the engine's 32-bit outputs (bucket rejection, as host_rng.h)
template <class Eng>
__device__ uint32_t uniform_draw(Eng& e, uint32_t range, int* draws) {
    if (range == 0) return 0;
    uint32_t bucket = 0xFFFFFFFFu / (range + 1u);
    if (0xFFFFFFFFu % (range + 1u) == range) ++bucket;
    for (;;) {
        (*draws)++;
        const uint32_t r = e.next() / bucket;
        if (r <= range) return r;
    }
}

// One sample with the full generators (rare: more than 226 draws from a Sampler).
__device__ __noinline__ bool pixel_uniform_slow(uint32_t sx, uint32_t sy, int W, int H, const uint8_t* lab,
                                               const uint8_t* ignored, int* x_out, int* y_out) {
    MtFull ex(sx), ey(sy);
    int dx = 0, dy = 0;
    for (long long tries = 0; tries < 100000000LL; tries++) {
        const int x = static_cast<int>(uniform_draw(ex, static_cast<uint32_t>(W - 1), &dx));
        const int y = static_cast<int>(uniform_draw(ey, static_cast<uint32_t>(H - 1), &dy));
        if (!ignored[lab[static_cast<long long>(y) * W + x]]) {
            *x_out = x;
            *y_out = y;
            return true;
        }
    }
    return false;
}

__global__ void pixel_uniform_kernel(const uint8_t* __restrict__ labels, const uint16_t* __restrict__ depth,
                                     const int* __restrict__ images, const int* __restrict__ draw_image,
                                     long long n, int W, int H, long long seed0, const uint8_t* __restrict__ ignored,
                                     uint8_t flip, cf_sample* __restrict__ out, unsigned long long* __restrict__ key,
                                     uint32_t* __restrict__ order, int* __restrict__ failed) {
    const long long plane = static_cast<long long>(W) * H;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int k = draw_image[i];
        const uint8_t* lab = labels + static_cast<long long>(images[k]) * plane;
        // the Samplers of sample i take seeds seed0 + 2i (x) and seed0 + 2i + 1 (y), as int wraps
        const uint32_t sx = static_cast<uint32_t>(seed0 + 2 * i), sy = static_cast<uint32_t>(seed0 + 2 * i + 1);
        MtHead ex(sx), ey(sy);
        int dx = 0, dy = 0, x = 0, y = 0;
        bool found = false;
        while (dx < 200 && dy < 200) {   // each loop draws at most a few values from each Sampler
            x = static_cast<int>(uniform_draw(ex, static_cast<uint32_t>(W - 1), &dx));
            y = static_cast<int>(uniform_draw(ey, static_cast<uint32_t>(H - 1), &dy));
            if (dx > 226 || dy > 226) break;
            if (!ignored[lab[static_cast<long long>(y) * W + x]]) {
                found = true;
                break;
            }
        }
        if (!found && !pixel_uniform_slow(sx, sy, W, H, lab, ignored, &x, &y)) {
            atomicOr(failed, 1);
            continue;
        }
        const long long p = static_cast<long long>(y) * W + x;
        const uint8_t label = lab[p];
        const uint16_t mm = depth[static_cast<long long>(images[k]) * plane + p];
        cf_sample s;
        s.x = static_cast<uint16_t>(x);
        s.y = static_cast<uint16_t>(y);
        s.image = static_cast<uint32_t>(k);
        s.depth = mm > 0 ? __fdiv_rn(static_cast<float>(static_cast<int>(mm)), 1000.0f) : 0.0f;
        s.label = label;
        s.flip = flip;
        s.reserved = 0;
        out[i] = s;
        // RandomTreeImage::train's block sort (random_tree_image.cpp:776-802): stable, in blocks of
        // 200000 samples, by (image, label, y/10, x/10)
        key[i] = (static_cast<unsigned long long>(i / 200000) << 48) | (static_cast<unsigned long long>(k) << 32) |
                 (static_cast<unsigned long long>(label) << 24) | (static_cast<unsigned long long>(y / 10) << 12) |
                 static_cast<unsigned long long>(x / 10);
        order[i] = static_cast<uint32_t>(i);
    }
}

__global__ void gather_samples_kernel(const cf_sample* __restrict__ in, const uint32_t* __restrict__ order,
                                      long long n, cf_sample* __restrict__ out) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = in[order[i]];
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
    CF_REQUIRE(images.size() < (1u << 16) && fr.W <= 40950 && fr.H <= 40950, "device sampling: frames too large");
    std::vector<uint8_t> classes;   // the sampled classes, ascending
    for (int c = 0; c < C; c++)
        if (!ign[c]) classes.push_back(static_cast<uint8_t>(c));
    fr.class_count.reserve(256);
    fr.class_start.reserve(256);
    std::vector<uint32_t> ccount(256, 0);
    unsigned long long n = 0;
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
        CF_CUDA_CHECK(cudaMemcpyAsync(&n, fr.count.get(), sizeof(n), cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        if (n > capacity) continue;   // more survivors than room: retry with a larger buffer
        CF_REQUIRE(n < (1ull << 31), "device sampling: too many candidates");
        fr.idx_a.reserve(n + 1);
        fr.idx_b.reserve(n + 1);
        fr.key_a.reserve(n + 1);
        fr.key_b.reserve(n + 1);
        CF_CUDA_CHECK(cudaMemsetAsync(fr.class_count.get(), 0, sizeof(uint32_t) * 256, st));
        launch_on(ctx, st, "sample_pairs", dim3(grid), dim3(256), 0, candidate_pairs_kernel,
                  reinterpret_cast<const uint4*>(d_cand), n, fr.idx_a.get(), fr.key_a.get(), fr.class_count.get());
        CF_CUDA_CHECK(cudaMemcpyAsync(ccount.data(), fr.class_count.get(), sizeof(uint32_t) * 256, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        bool enough = true;
        for (uint8_t c : classes)
            if (ccount[c] < per_class) enough = false;
        if (enough) break;
    }
    // (class, key, pixel) order: a stable sort by pixel index (the candidates were appended in any
    // order), then a stable sort by (class << 32 | key)
    const int ni = static_cast<int>(n);
    const unsigned long long n_sel = static_cast<unsigned long long>(per_class) * classes.size();
    size_t t1 = 0, t2 = 0, t3 = 0;
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, t1, fr.idx_a.get(), fr.idx_b.get(), fr.key_a.get(),
                                                  fr.key_b.get(), ni, 0, 32, st));
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, t2, fr.key_b.get(), fr.key_a.get(), fr.idx_b.get(),
                                                  fr.idx_a.get(), ni, 0, 40, st));
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, t3, fr.key_b.get(), fr.key_a.get(), fr.idx_b.get(),
                                                  fr.idx_a.get(), static_cast<int>(n_sel), 0, 64, st));
    const size_t temp = std::max(t1, std::max(t2, t3));
    if (fr.sort_temp.capacity() < temp) {
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        fr.sort_temp.reserve(temp);
    }
    size_t tb = temp;
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(fr.sort_temp.get(), tb, fr.idx_a.get(), fr.idx_b.get(),
                                                  fr.key_a.get(), fr.key_b.get(), ni, 0, 32, st));
    tb = temp;
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(fr.sort_temp.get(), tb, fr.key_b.get(), fr.key_a.get(),
                                                  fr.idx_b.get(), fr.idx_a.get(), ni, 0, 40, st));
    // every class's first per_class candidates, keyed by the block order
    std::vector<uint32_t> start(256, 0);
    for (int c = 1; c < 256; c++) start[c] = start[c - 1] + ccount[c - 1];
    CF_CUDA_CHECK(cudaMemcpyAsync(fr.class_start.get(), start.data(), sizeof(uint32_t) * 256, cudaMemcpyHostToDevice, st));
    CF_CUDA_CHECK(cudaMemcpyAsync(fr.ignored.get(), classes.data(), classes.size(), cudaMemcpyHostToDevice, st));
    launch_on(ctx, st, "sample_select", dim3(grid), dim3(256), 0, select_kernel, fr.idx_a.get(), fr.class_start.get(),
              fr.ignored.get(), static_cast<int>(classes.size()), static_cast<unsigned long long>(per_class), plane,
              fr.W, fr.key_b.get(), fr.idx_b.get());
    tb = temp;
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(fr.sort_temp.get(), tb, fr.key_b.get(), fr.key_a.get(),
                                                  fr.idx_b.get(), fr.idx_a.get(), static_cast<int>(n_sel), 0, 64, st));
    fr.out.reserve(n_sel + 1);
    launch_on(ctx, st, "sample_emit", dim3(grid), dim3(256), 0, emit_samples_kernel, fr.key_a.get(), fr.idx_a.get(),
              n_sel, fr.images.get(), fr.depth.get(), plane, fr.W, flip, fr.out.get());
    std::vector<cf_sample> out(n_sel);
    CF_CUDA_CHECK(cudaMemcpyAsync(out.data(), fr.out.get(), sizeof(cf_sample) * n_sel, cudaMemcpyDeviceToHost, st));
    CF_CUDA_CHECK(cudaStreamSynchronize(st));
    (void)depth_host;
    return out;
}

std::vector<cf_sample> sample_pixel_uniform_device(cf_context* ctx, DeviceFrames& fr, const std::vector<int>& images,
                                                   int C, const uint8_t* ignored_host, int subsample_count,
                                                   RandomSource& rs, uint8_t flip, std::vector<uint32_t>* prior) {
    const long long n = static_cast<long long>(subsample_count) * static_cast<long long>(images.size());
    CF_REQUIRE(n > 0 && n < (1LL << 31), "device pixelUniform sampling: sample count out of range");
    CF_REQUIRE(images.size() < (1u << 16) && fr.W <= 40950 && fr.H <= 40950 && n / 200000 < (1LL << 16),
               "device pixelUniform sampling: frames too large");
    std::vector<uint8_t> ign(256, 0);
    bool all_ignored = true;
    for (int c = 0; c < 256; c++) {
        if (ignored_host && ignored_host[c]) ign[c] = 1;
    }
    for (int c = 0; c < 256; c++) all_ignored = all_ignored && ign[c];
    CF_REQUIRE(!all_ignored, "no classes left to sample");
    // the image of every sample: one Sampler over the image list, drawn in sequence (host)
    Sampler rgen_image = rs.uniform(static_cast<int>(images.size()));
    std::vector<int> draw(static_cast<size_t>(n));
    for (long long i = 0; i < n; i++) draw[i] = rgen_image.next();
    // the x and y Samplers of every sample take the next 2n seeds of the tree's random source
    const long long seed0 = *rs.counter;
    *rs.counter = static_cast<int32_t>(static_cast<uint32_t>(seed0 + 2 * n));
    cudaStream_t st = fr.stream;
    CF_REQUIRE(st != nullptr && images.size() <= static_cast<size_t>(fr.n), "device sampling: frames not uploaded");
    fr.idx_a.reserve(n + 1);
    fr.idx_b.reserve(n + 1);
    fr.key_a.reserve(n + 1);
    fr.key_b.reserve(n + 1);
    fr.out.reserve(2 * n + 1);
    fr.class_start.reserve(256);
    CF_CUDA_CHECK(cudaMemcpyAsync(fr.images.get(), images.data(), sizeof(int) * images.size(), cudaMemcpyHostToDevice, st));
    CF_CUDA_CHECK(cudaMemcpyAsync(fr.ignored.get(), ign.data(), 256, cudaMemcpyHostToDevice, st));
    CF_CUDA_CHECK(cudaMemcpyAsync(fr.idx_b.get(), draw.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    CF_CUDA_CHECK(cudaMemsetAsync(fr.bad.get(), 0, sizeof(int), st));
    const int grid = ctx->num_sms * 8;
    {
        // class prior of the listed images (calculateLabelPriorDistribution, random_tree_image.cpp:885-909)
        const long long plane = static_cast<long long>(fr.W) * fr.H;
        fr.counts.reserve(512);
        CF_CUDA_CHECK(cudaMemsetAsync(fr.counts.get(), 0, sizeof(uint32_t) * 2 * C, st));
        launch_on(ctx, st, "sample_counts", dim3(grid), dim3(256), 0, tree_pixel_counts_kernel, fr.labels.get(),
                  fr.depth.get(), fr.images.get(), plane, plane * static_cast<long long>(images.size()), C,
                  fr.ignored.get(), fr.counts.get(), fr.counts.get() + C, fr.bad.get());
        std::vector<uint32_t> counts(2 * C);
        int bad = 0;
        CF_CUDA_CHECK(cudaMemcpyAsync(counts.data(), fr.counts.get(), sizeof(uint32_t) * 2 * C, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(&bad, fr.bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        CF_REQUIRE(!bad, "label image holds a label >= number of classes");
        if (prior) prior->assign(counts.begin(), counts.begin() + C);
    }
    cf_sample* raw = fr.out.get() + n;
    launch_on(ctx, st, "sample_pixel_uniform", dim3(grid), dim3(128), 0, pixel_uniform_kernel, fr.labels.get(),
              fr.depth.get(), fr.images.get(), reinterpret_cast<const int*>(fr.idx_b.get()), n, fr.W, fr.H, seed0,
              fr.ignored.get(), flip, raw, fr.key_a.get(), fr.idx_a.get(), fr.bad.get());
    size_t temp = 0;
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, temp, fr.key_a.get(), fr.key_b.get(), fr.idx_a.get(),
                                                  fr.idx_b.get(), static_cast<int>(n), 0, 64, st));
    if (fr.sort_temp.capacity() < temp) {
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        fr.sort_temp.reserve(temp);
    }
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(fr.sort_temp.get(), temp, fr.key_a.get(), fr.key_b.get(),
                                                  fr.idx_a.get(), fr.idx_b.get(), static_cast<int>(n), 0, 64, st));
    launch_on(ctx, st, "sample_gather", dim3(grid), dim3(256), 0, gather_samples_kernel, raw, fr.idx_b.get(), n,
              fr.out.get());
    std::vector<cf_sample> out(static_cast<size_t>(n));
    int failed = 0;
    CF_CUDA_CHECK(cudaMemcpyAsync(out.data(), fr.out.get(), sizeof(cf_sample) * n, cudaMemcpyDeviceToHost, st));
    CF_CUDA_CHECK(cudaMemcpyAsync(&failed, fr.bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    CF_CUDA_CHECK(cudaStreamSynchronize(st));
    CF_REQUIRE(!failed, "pixelUniform sampling found no usable pixel");
    return out;
}

}  // namespace cf
