// RandomForestImage::train (random_forest_image.cpp:132-182) on raw host frames: integral images
// on the GPU, the per-tree random source, the maxImages reservoir, the class prior, training-pixel
// sampling on the host (classUniform / pixelUniform, random_tree_image.cpp:840-1059), the block
// sort of the samples (random_tree_image.cpp:776-802) and GPU tree training.
//
// Sampling runs on one host thread: the reference's multi-threaded class-uniform sampling merges
// per-thread reservoirs in completion order and is not reproducible; with one thread it is.
// The block sort orders by (image position in the tree's image list, label, y/10, x/10) with a
// stable sort; the reference sorts by image address with std::sort, whose tie order is unspecified.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <memory>

#include "host_rng.h"
#include "sampling.h"
#include "split_eval.h"
#include "tree.h"

namespace cf {

cf_tree* train_tree(cf_dataset* ds, const cf_sample* samples, int N, int C, const cf_train_config& cfg, int tree_id,
                    int32_t* seed_counter, int mode, const LevelEvaluator::Shard* shard = nullptr);

namespace {

struct Reservoir {
    size_t count = 0;
    std::vector<cf_sample> items;
};

// ReservoirSampler::sample (random_tree.h:1085-1105)
inline void reservoir_add(Reservoir& r, size_t capacity, Sampler& sampler, const cf_sample& s) {
    if (r.items.size() < capacity) {
        r.items.push_back(s);
    } else {
        const size_t rnd = static_cast<size_t>(sampler.next()) % (r.count + 1);
        if (rnd < capacity) r.items[rnd] = s;
    }
    r.count++;
}

inline cf_sample make_sample(int img, int x, int y, uint16_t depth_mm, uint8_t label, uint8_t flip) {
    cf_sample s;
    s.x = static_cast<uint16_t>(x);
    s.y = static_cast<uint16_t>(y);
    s.image = static_cast<uint32_t>(img);
    s.depth = depth_mm > 0 ? static_cast<float>(static_cast<int>(depth_mm)) / 1000.0f : 0.0f;
    s.label = label;
    s.flip = flip;
    s.reserved = 0;
    return s;
}

std::vector<cf_sample> sample_class_uniform(const std::vector<int>& images, int W, int H, const uint8_t* labels,
                                            const uint16_t* depth, int C, const uint8_t* ignored, int subsample_count,
                                            RandomSource& rs, uint8_t flip) {
    int numLabels = C;
    for (int c = 0; c < C; c++)
        if (ignored && ignored[c]) numLabels--;
    CF_REQUIRE(numLabels > 0, "no classes left to sample");
    const size_t per_class = static_cast<size_t>(
        std::ceil(images.size() * static_cast<double>(subsample_count) / static_cast<double>(numLabels)));
    const int randomSeed = rs.uniform(0xFFFFFF).next();
    std::vector<Reservoir> res(C);
    int32_t chunk_counter = randomSeed;
    RandomSource chunk_rs(&chunk_counter);
    Sampler sampler = chunk_rs.uniform(0x7FFFFFFF);
    const size_t plane = static_cast<size_t>(W) * H;
    for (size_t k = 0; k < images.size(); k++) {
        const int img = images[k];
        const uint8_t* L = labels + plane * img;
        const uint16_t* D = depth + plane * img;
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const size_t p = static_cast<size_t>(y) * W + x;
                const uint8_t label = L[p];
                CF_REQUIRE(label < C, "label image holds a label >= number of classes");
                if (ignored && ignored[label]) continue;
                if (D[p] == 0) continue;
                reservoir_add(res[label], per_class, sampler, make_sample(static_cast<int>(k), x, y, D[p], label, flip));
            }
    }
    (void)rs.uniform(0x7FFFFFFF);  // merge sampler; with one chunk it draws nothing
    std::vector<cf_sample> all;
    for (int label = 0; label < C; label++) {
        if (ignored && ignored[label]) continue;
        all.insert(all.begin(), res[label].items.begin(), res[label].items.end());
    }
    CF_REQUIRE(all.size() == per_class * numLabels, "failed to sample enough pixels");
    return all;
}

std::vector<cf_sample> sample_pixel_uniform(const std::vector<int>& images, int W, int H, const uint8_t* labels,
                                            const uint16_t* depth, const uint8_t* ignored, int subsample_count,
                                            RandomSource& rs, uint8_t flip) {
    Sampler rgen_image = rs.uniform(static_cast<int>(images.size()));
    std::vector<cf_sample> out;
    const size_t plane = static_cast<size_t>(W) * H;
    const size_t total = static_cast<size_t>(subsample_count) * images.size();
    for (size_t n = 0; n < total; n++) {
        const int k = rgen_image.next();
        Sampler rx = rs.uniform(W);
        Sampler ry = rs.uniform(H);
        const int img = images[k];
        for (int tries = 0;; tries++) {
            CF_REQUIRE(tries < 100000000, "pixelUniform sampling found no usable pixel");
            const int x = rx.next(), y = ry.next();
            const size_t p = plane * img + static_cast<size_t>(y) * W + x;
            const uint8_t label = labels[p];
            if (ignored && ignored[label]) continue;
            out.push_back(make_sample(k, x, y, depth[p], label, flip));
            break;
        }
    }
    return out;
}

// RandomTreeImage::train block sort (random_tree_image.cpp:776-802), stable
void block_sort(std::vector<cf_sample>& s) {
    const size_t block = 200000;
    for (size_t b = 0; b < s.size(); b += block) {
        const size_t e = std::min(s.size(), b + block);
        std::stable_sort(s.begin() + b, s.begin() + e, [](const cf_sample& a, const cf_sample& c) {
            if (a.image != c.image) return a.image < c.image;
            if (a.label != c.label) return a.label < c.label;
            if (a.y / 10 != c.y / 10) return a.y / 10 < c.y / 10;
            if (a.x / 10 != c.x / 10) return a.x / 10 < c.x / 10;
            return false;
        });
    }
}

}  // namespace

// Training pixels of one tree as RandomForestImage::train / RandomTreeImage::train draw them:
// image reservoir (maxImages), class prior, sampling, block sort. Sample image indices refer to
// the dataset. `rs` is the tree's random source (seed SEED + treeId).
// With `frames` (config.sampler == 1, classUniform) the class prior and the sampling run on the
// device (sample_class_uniform_device).
std::vector<cf_sample> sample_tree(int num_images, int width, int height, const uint8_t* labels,
                                   const uint16_t* depth_mm, int num_classes, const uint8_t* ignored,
                                   const cf_train_config& config, int num_trees, RandomSource& rs,
                                   std::vector<uint32_t>& prior, cf_context* ctx = nullptr,
                                   DeviceFrames* frames = nullptr) {
    const size_t plane = static_cast<size_t>(width) * height;
    std::vector<int> images(num_images);
    for (int i = 0; i < num_images; i++) images[i] = i;
    if (config.max_images > 0 && num_images > config.max_images) {
        Sampler sampler = rs.uniform(0, 10 * num_images);
        std::vector<int> res;
        size_t count = 0;
        for (int i = 0; i < num_images; i++) {
            if (res.size() < static_cast<size_t>(config.max_images)) {
                res.push_back(i);
            } else {
                const size_t rnd = static_cast<size_t>(sampler.next()) % (count + 1);
                if (rnd < static_cast<size_t>(config.max_images)) res[rnd] = i;
            }
            count++;
        }
        images = res;
    }
    const int subsample = static_cast<int>(config.samples_per_image / static_cast<uint32_t>(num_trees));
    CF_REQUIRE(subsample > 0, "samplesPerImage / treeCount must be > 0");
    const uint8_t flip = config.horizontal_flipping ? 2 : 0;
    if (frames && config.sampler == 1) {
        std::vector<cf_sample> samples =
            config.subsampling_type == 0
                ? sample_class_uniform_device(ctx, *frames, images, depth_mm, num_classes, ignored, subsample, rs, flip,
                                              &prior)
                : sample_pixel_uniform_device(ctx, *frames, images, num_classes, ignored, subsample, rs, flip, &prior);
        for (auto& s : samples) s.image = static_cast<uint32_t>(images[s.image]);
        return samples;
    }
    // calculateLabelPriorDistribution (random_tree_image.cpp:885-909)
    prior.assign(num_classes, 0);
    for (int img : images)
        for (size_t p = 0; p < plane; p++) {
            const uint8_t l = labels[plane * img + p];
            CF_REQUIRE(l < num_classes, "label image holds a label >= number of classes");
            prior[l]++;
        }
    std::vector<cf_sample> samples =
        config.subsampling_type == 0
            ? sample_class_uniform(images, width, height, labels, depth_mm, num_classes, ignored, subsample, rs, flip)
            : sample_pixel_uniform(images, width, height, labels, depth_mm, ignored, subsample, rs, flip);
    block_sort(samples);
    for (auto& s : samples) s.image = static_cast<uint32_t>(images[s.image]);
    return samples;
}

}  // namespace cf

using namespace cf;

extern "C" {

cf_status cf_forest_seed(int32_t random_seed, int32_t* seed) {
    return guard([&] {
        CF_REQUIRE(seed, "cf_forest_seed: NULL argument");
        int32_t counter = random_seed;
        RandomSource rs(&counter);
        *seed = rs.uniform(0xFFFF).next();
    });
}

cf_status cf_sample_tree_pixels(int num_images, int width, int height, const uint8_t* labels, const uint16_t* depth_mm,
                                int num_classes, const uint8_t* ignored, const cf_train_config* config, int num_trees,
                                int32_t* seed_counter, cf_sample* out, int64_t capacity, int64_t* count,
                                uint32_t* prior) {
    return guard([&] {
        CF_REQUIRE(labels && depth_mm && config && seed_counter && count, "cf_sample_tree_pixels: NULL argument");
        CF_REQUIRE(num_images >= 1 && width >= 1 && height >= 1, "cf_sample_tree_pixels: empty input");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_sample_tree_pixels: classes must be in [1, 256]");
        CF_REQUIRE(num_trees >= 1, "cf_sample_tree_pixels: need at least one tree");
        RandomSource rs(seed_counter);
        std::vector<uint32_t> pr;
        std::vector<cf_sample> s = sample_tree(num_images, width, height, labels, depth_mm, num_classes, ignored,
                                               *config, num_trees, rs, pr);
        *count = static_cast<int64_t>(s.size());
        if (out) {
            CF_REQUIRE(capacity >= static_cast<int64_t>(s.size()), "cf_sample_tree_pixels: output buffer too small");
            std::memcpy(out, s.data(), sizeof(cf_sample) * s.size());
        }
        if (prior) std::memcpy(prior, pr.data(), sizeof(uint32_t) * pr.size());
    });
}

cf_status cf_sample_tree_pixels_device(cf_context* ctx, int num_images, int width, int height, const uint8_t* labels,
                                       const uint16_t* depth_mm, int num_classes, const uint8_t* ignored,
                                       const cf_train_config* config, int num_trees, int32_t* seed_counter,
                                       cf_sample* out, int64_t capacity, int64_t* count, uint32_t* prior) {
    return guard([&] {
        CF_REQUIRE(ctx && labels && depth_mm && config && seed_counter && count,
                   "cf_sample_tree_pixels_device: NULL argument");
        CF_REQUIRE(num_images >= 1 && width >= 1 && height >= 1, "cf_sample_tree_pixels_device: empty input");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_sample_tree_pixels_device: classes must be in [1, 256]");
        CF_REQUIRE(num_trees >= 1, "cf_sample_tree_pixels_device: need at least one tree");
        CF_REQUIRE(config->subsampling_type == 0 || config->subsampling_type == 1,
                   "cf_sample_tree_pixels_device: unknown subsamplingType");
        make_current(ctx);
        DeviceFrames frames;
        frames.upload(ctx, num_images, width, height, labels, depth_mm);
        cf_train_config cfg = *config;
        cfg.sampler = 1;
        RandomSource rs(seed_counter);
        std::vector<uint32_t> pr;
        std::vector<cf_sample> s = sample_tree(num_images, width, height, labels, depth_mm, num_classes, ignored, cfg,
                                               num_trees, rs, pr, ctx, &frames);
        *count = static_cast<int64_t>(s.size());
        if (out) {
            CF_REQUIRE(capacity >= static_cast<int64_t>(s.size()), "cf_sample_tree_pixels_device: output buffer too small");
            std::memcpy(out, s.data(), sizeof(cf_sample) * s.size());
        }
        if (prior) std::memcpy(prior, pr.data(), sizeof(uint32_t) * pr.size());
    });
}

cf_status cf_forest_train(cf_context* ctx, int num_images, int width, int height, const uint8_t* rgb,
                          const uint16_t* depth_mm, const uint8_t* labels, int num_classes, const uint8_t* ignored,
                          const cf_train_config* config, int num_trees, int mode, cf_tree** trees) {
    return guard([&] {
        CF_REQUIRE(ctx && rgb && depth_mm && labels && config && trees, "cf_forest_train: NULL argument");
        CF_REQUIRE(num_images >= 1, "no training images");
        CF_REQUIRE(num_trees >= 1, "cf_forest_train: need at least one tree");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_forest_train: classes must be in [1, 256]");
        CF_REQUIRE(config->subsampling_type == 0 || config->subsampling_type == 1, "unknown subsamplingType");
        make_current(ctx);
        for (int t = 0; t < num_trees; t++) trees[t] = nullptr;
        cf_dataset* ds_raw = nullptr;
        {
            const cf_status st = cf_dataset_create(ctx, num_images, width, height, &ds_raw);
            if (st != CF_OK) fail(st, "cf_forest_train: dataset allocation failed");
        }
        std::unique_ptr<cf_dataset, cf_status (*)(cf_dataset*)> ds(ds_raw, cf_dataset_destroy);
        // useDepthFilling: the filled depth frames serve the integral images and the sampling
        std::vector<uint16_t> filled;
        if (config->use_depth_filling) {
            filled.assign(depth_mm, depth_mm + static_cast<size_t>(num_images) * width * height);
            const cf_status st = cf_fill_depth(ctx, num_images, width, height, filled.data(), 0);
            if (st != CF_OK) fail(st, "cf_forest_train: depth filling failed");
            depth_mm = filled.data();
        }
        {
            const cf_status st =
                cf_dataset_upload_raw_ex(ds.get(), 0, num_images, rgb, depth_mm, 0, 0, config->use_cie_lab ? 1 : 0);
            if (st != CF_OK) fail(st, "cf_forest_train: upload failed");
        }
        // RandomForestImage::train: SEED from the configured seed, tree seed SEED + treeId
        int32_t SEED = 0;
        {
            const cf_status st = cf_forest_seed(config->random_seed, &SEED);
            if (st != CF_OK) fail(st, "cf_forest_train: seed");
        }
        CF_REQUIRE(config->sampler == 0 || config->sampler == 1, "unknown sampler");
        std::unique_ptr<DeviceFrames> frames;
        if (config->sampler == 1) {
            frames.reset(new DeviceFrames());
            frames->upload(ctx, num_images, width, height, labels, depth_mm);
        }
        // the training pixels of tree t + 1 are drawn on a host thread (and the sampler's own stream)
        // while tree t trains
        struct Drawn {
            std::vector<cf_sample> samples;
            std::vector<uint32_t> prior;
            int32_t counter = 0;
        };
        auto draw = [&](int t) {
            CF_CUDA_CHECK(cudaSetDevice(ctx->device));
            Drawn d;
            d.counter = SEED + t;
            RandomSource rs(&d.counter);
            d.samples = sample_tree(num_images, width, height, labels, depth_mm, num_classes, ignored, *config,
                                    num_trees, rs, d.prior, ctx, frames.get());
            return d;
        };
        try {
            std::future<Drawn> next = std::async(std::launch::async, draw, 0);
            for (int t = 0; t < num_trees; t++) {
                Drawn cur = next.get();
                if (t + 1 < num_trees) next = std::async(std::launch::async, draw, t + 1);
                cf_tree* tree = train_tree(ds.get(), cur.samples.data(), static_cast<int>(cur.samples.size()),
                                           num_classes, *config, t, &cur.counter, mode);
                tree->prior = cur.prior;
                trees[t] = tree;
            }
        } catch (...) {
            for (int t = 0; t < num_trees; t++) {
                delete trees[t];
                trees[t] = nullptr;
            }
            throw;
        }
    });
}

cf_status cf_tree_prior(cf_tree* tree, uint32_t* prior, int capacity, int* count) {
    return guard([&] {
        CF_REQUIRE(tree, "cf_tree_prior: tree is NULL");
        if (count) *count = static_cast<int>(tree->prior.size());
        if (prior) {
            CF_REQUIRE(capacity >= static_cast<int>(tree->prior.size()), "cf_tree_prior: buffer too small");
            std::memcpy(prior, tree->prior.data(), sizeof(uint32_t) * tree->prior.size());
        }
    });
}

cf_status cf_tree_set_prior(cf_tree* tree, const uint32_t* prior, int count) {
    return guard([&] {
        CF_REQUIRE(tree && prior, "cf_tree_set_prior: NULL argument");
        CF_REQUIRE(count == tree->C, "cf_tree_set_prior: prior needs one entry per class");
        tree->prior.assign(prior, prior + count);
    });
}

}  // extern "C"
