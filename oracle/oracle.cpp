/*
 * CPU oracle for the CURFIL hot path. TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Built with -ffp-contract=off and without -ffast-math so that every floating-point
 * operation rounds exactly as the reference's host build (x86-64 SSE, no FMA) does.
 */
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <stdexcept>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double kNaN = std::numeric_limits<double>::quiet_NaN();

/* ------------------------------------------------------------------------------------------
 * Random numbers of the reference host code
 * ---------------------------------------------------------------------------------------- */

/* boost::uniform_int<> over an mt19937 (Boost.Random generate_uniform_int, integral engine
 * branch): the engine's range 2^32-1 is split into buckets of equal size and draws that fall
 * past the last whole bucket are rejected. Restated from the published Boost algorithm. */
int32_t uniform_int_draw(std::mt19937& eng, int32_t lo, int32_t hi) {
    const uint32_t range = static_cast<uint32_t>(hi) - static_cast<uint32_t>(lo);
    const uint32_t brange = 0xFFFFFFFFu;
    if (range == 0) return lo;
    if (range == brange) return static_cast<int32_t>(static_cast<uint32_t>(eng()) + static_cast<uint32_t>(lo));
    uint32_t bucket = brange / (range + 1u);
    if (brange % (range + 1u) == range) ++bucket;
    for (;;) {
        const uint32_t r = static_cast<uint32_t>(eng()) / bucket;
        if (r <= range) return static_cast<int32_t>(r + static_cast<uint32_t>(lo));
    }
}

/* Sampler (random_tree.h:1009-1063): fresh mt19937(seed) + uniform_int(lo, hi). */
struct Sampler {
    std::mt19937 eng;
    int32_t lo, hi;
    Sampler(int seed, int lo_, int hi_) : eng(static_cast<uint32_t>(seed)), lo(lo_), hi(hi_) {}
    int32_t next() { return uniform_int_draw(eng, lo, hi); }
};

/* RandomSource::uniformSampler (random_tree.h:1129-1156): every sampler takes seed++. */
Sampler uniform_sampler(int* seed_counter, int upper_exclusive) {
    return Sampler((*seed_counter)++, 0, upper_exclusive - 1);
}

/* ------------------------------------------------------------------------------------------
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11). Stands in for the cuRAND XORWOW stream of generateRandomFeaturesKernel.
 * ---------------------------------------------------------------------------------------- */
void philox4x32_10(uint32_t k0, uint32_t k1, uint32_t c[4]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        const uint64_t p0 = static_cast<uint64_t>(M0) * c[0];
        const uint64_t p1 = static_cast<uint64_t>(M1) * c[2];
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

/* Per-feature stream: key (seed, feature), counter (block, 0, 0, 0), words used in order. */
struct FeatureStream {
    uint32_t key0, key1, block = 0, pos = 4;
    uint32_t buf[4];
    FeatureStream(uint32_t seed, uint32_t feat) : key0(seed), key1(feat) {}
    uint32_t next_u32() {
        if (pos == 4) {
            buf[0] = block++;
            buf[1] = buf[2] = buf[3] = 0;
            philox4x32_10(key0, key1, buf);
            pos = 0;
        }
        return buf[pos++];
    }
    /* uniform float in (0, 1], exact: ((u >> 8) + 1) * 2^-24 (same range as curand_uniform) */
    float uniform() { return static_cast<float>((next_u32() >> 8) + 1u) * (1.0f / 16777216.0f); }
};

/* ------------------------------------------------------------------------------------------
 * Image access
 * ---------------------------------------------------------------------------------------- */
inline const float* color_plane(const orc_dataset* ds, int image, int channel) {
    const size_t hw = static_cast<size_t>(ds->width) * ds->height;
    return ds->color + (static_cast<size_t>(image) * 3 + channel) * hw;
}
inline size_t pix(const orc_dataset* ds, int image, int x, int y) {
    return static_cast<size_t>(image) * ds->width * ds->height + static_cast<size_t>(y) * ds->width + x;
}

/* XY::normalize (random_tree_image.h:82-87): int / float -> float division, truncation. */
inline int normalize_coord(int v, float depth) { return static_cast<int>(static_cast<float>(v) / depth); }

/* PixelInstance::averageRegionDepth (random_tree_image.h:268-316) */
double average_region_depth(const orc_dataset* ds, const orc_sample* s, int ox, int oy, int rx, int ry) {
    const int width = std::max(1, rx);
    const int height = std::max(1, ry);
    const int x = s->x + ox;
    const int y = s->y + oy;
    const int leftX = x - width, rightX = x + width, upperY = y - height, lowerY = y + height;
    if (leftX < 0 || rightX >= ds->width || upperY < 0 || lowerY >= ds->height) return kNaN;
    const int img = static_cast<int>(s->image);
    const int32_t ulv = ds->depth_valid[pix(ds, img, leftX, upperY)];
    const int32_t urv = ds->depth_valid[pix(ds, img, rightX, upperY)];
    const int32_t lrv = ds->depth_valid[pix(ds, img, rightX, lowerY)];
    const int32_t llv = ds->depth_valid[pix(ds, img, leftX, lowerY)];
    const int numValid = (lrv - urv) + (ulv - llv);
    if (numValid == 0) return kNaN;
    const int64_t lr = ds->depth_sum[pix(ds, img, rightX, lowerY)];
    const int64_t ll = ds->depth_sum[pix(ds, img, leftX, lowerY)];
    const int64_t ur = ds->depth_sum[pix(ds, img, rightX, upperY)];
    const int64_t ul = ds->depth_sum[pix(ds, img, leftX, upperY)];
    const int64_t sum = (lr - ur) + (ul - ll);
    const double feat = static_cast<double>(sum) / 1000.0;
    return feat / numValid;
}

/* PixelInstance::averageRegionColor (random_tree_image.h:222-262) */
double average_region_color(const orc_dataset* ds, const orc_sample* s, int ox, int oy, int rx, int ry,
                            int channel) {
    const int width = std::max(1, rx);
    const int height = std::max(1, ry);
    const int x = s->x + ox;
    const int y = s->y + oy;
    const int leftX = x - width, rightX = x + width, upperY = y - height, lowerY = y + height;
    if (leftX < 0 || rightX >= ds->width || upperY < 0 || lowerY >= ds->height) return kNaN;
    const float* plane = color_plane(ds, static_cast<int>(s->image), channel);
    const double lr = plane[static_cast<size_t>(lowerY) * ds->width + rightX];
    const double ll = plane[static_cast<size_t>(lowerY) * ds->width + leftX];
    const double ur = plane[static_cast<size_t>(upperY) * ds->width + rightX];
    const double ul = plane[static_cast<size_t>(upperY) * ds->width + leftX];
    if (std::isnan(lr) || std::isnan(ll) || std::isnan(ur) || std::isnan(ul)) return kNaN;
    return (lr - ur) + (ul - ll);
}

/* calculateDepthFeature / calculateColorFeature (random_tree_image.h:564-623) */
double feature_response(const orc_dataset* ds, const orc_sample* s, const int8_t* f, bool flip) {
    const float depth = s->depth;
    if (!(depth > 0.0f)) return kNaN; /* Depth::isValid(): value > 0 */
    const int type = f[0];
    int o1x = f[1], o1y = f[2], o2x = f[3], o2y = f[4];
    const int r1x = f[5], r1y = f[6], r2x = f[7], r2y = f[8];
    const int ch1 = static_cast<uint8_t>(f[9]), ch2 = static_cast<uint8_t>(f[10]);
    if (flip) {
        o1x = -o1x;
        o2x = -o2x;
    }
    const int n_o1x = normalize_coord(o1x, depth), n_o1y = normalize_coord(o1y, depth);
    const int n_r1x = normalize_coord(r1x, depth), n_r1y = normalize_coord(r1y, depth);
    const int n_o2x = normalize_coord(o2x, depth), n_o2y = normalize_coord(o2y, depth);
    const int n_r2x = normalize_coord(r2x, depth), n_r2y = normalize_coord(r2y, depth);
    double a, b;
    if (type == 0) { /* DEPTH */
        a = average_region_depth(ds, s, n_o1x, n_o1y, n_r1x, n_r1y);
        if (std::isnan(a)) return a;
        b = average_region_depth(ds, s, n_o2x, n_o2y, n_r2x, n_r2y);
        if (std::isnan(b)) return b;
    } else { /* COLOR */
        a = average_region_color(ds, s, n_o1x, n_o1y, n_r1x, n_r1y, ch1);
        if (std::isnan(a)) return a;
        b = average_region_color(ds, s, n_o2x, n_o2y, n_r2x, n_r2y, ch2);
        if (std::isnan(b)) return b;
    }
    return a - b;
}

inline void feature_column(const int8_t* features, int F, int f, int8_t out[11]) {
    for (int r = 0; r < 11; r++) out[r] = features[static_cast<size_t>(r) * F + f];
}

/* getSortKey (random_tree_image.h:444-452) */
int32_t sort_key(const int8_t f[11]) {
    int32_t key = 0;
    key |= static_cast<uint8_t>(f[0] & 0x03) << 30;
    key |= static_cast<uint8_t>(f[9] & 0x0F) << 26;
    key |= static_cast<uint8_t>(f[10] & 0x0F) << 22;
    key |= static_cast<uint8_t>((f[2] + 127) & 0xFF) << 14;
    key |= static_cast<uint8_t>((f[1] + 127) & 0xFF) << 6;
    return key;
}

/* InformationGainScore::entropy (score.h:51-56) */
inline double entropy(double p) { return p == 0.0 ? 0.0 : -p * std::log2(p); }

/* normalizeScore (score.h:62-77) */
inline double normalize_score(double s) {
    if (s > 1.0) return 1.0;
    if (s < 0.0) return 0.0;
    return s;
}

/* detail::isScoreBetter (random_tree.cpp:36-52) */
inline bool is_score_better(double best, double score) {
    const double diff = std::fabs(score - best);
    if (diff < 1e-13) return false;
    return score > best;
}

}  // namespace

extern "C" {

/* ------------------------------------------------------------------------------------------
 * Integral images (image.cpp:250-277): sequential row-major scan, one Kahan carry.
 * ---------------------------------------------------------------------------------------- */
void orc_integral_float_color(int width, int height, const float* color_in, float* color_out) {
    std::vector<double> data(static_cast<size_t>(width) * height);
    for (int c = 0; c < 3; c++) {
        const size_t base = static_cast<size_t>(c) * width * height;
        for (size_t i = 0; i < data.size(); i++) data[i] = color_in[base + i];
        double carry = 0.0;
        for (int y = 0; y < height; ++y) {
            const size_t prev = static_cast<size_t>(y - 1) * width;
            const size_t row = static_cast<size_t>(y) * width;
            for (int x = 0; x < width; ++x) {
                const double above = (y > 0) ? data[prev + x] : 0.0;
                const double left = (x > 0) ? data[row + x - 1] : 0.0;
                const double aboveLeft = (x > 0 && y > 0) ? data[prev + x - 1] : 0.0;
                const double dy = (left + above - aboveLeft) - carry;
                const double t = data[row + x] + dy;
                carry = (t - data[row + x]) - dy;
                data[row + x] = t;
            }
        }
        for (size_t i = 0; i < data.size(); i++) color_out[base + i] = static_cast<float>(data[i]);
    }
}

void orc_integral(int width, int height, const uint8_t* rgb, const uint16_t* depth_mm, float* color_out,
                  int64_t* depth_sum_out, int32_t* depth_valid_out) {
    const size_t hw = static_cast<size_t>(width) * height;
    std::vector<float> planes(3 * hw);
    for (size_t i = 0; i < hw; i++)
        for (int c = 0; c < 3; c++) planes[c * hw + i] = static_cast<float>(rgb[i * 3 + c]);
    orc_integral_float_color(width, height, planes.data(), color_out);
    /* depth channels: RGBDImage::setDepth stores 0 for invalid depth (image.h:344-350); the
     * integer scan is exact, so the Kahan carry stays zero. */
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            const size_t i = static_cast<size_t>(y) * width + x;
            const int64_t d = depth_mm[i];
            const int32_t v = d > 0 ? 1 : 0;
            const int64_t above = y > 0 ? depth_sum_out[i - width] : 0;
            const int64_t left = x > 0 ? depth_sum_out[i - 1] : 0;
            const int64_t al = (x > 0 && y > 0) ? depth_sum_out[i - width - 1] : 0;
            depth_sum_out[i] = d + left + above - al;
            const int32_t av = y > 0 ? depth_valid_out[i - width] : 0;
            const int32_t lv = x > 0 ? depth_valid_out[i - 1] : 0;
            const int32_t alv = (x > 0 && y > 0) ? depth_valid_out[i - width - 1] : 0;
            depth_valid_out[i] = v + lv + av - alv;
        }
    }
}

float orc_pixel_depth(const orc_dataset* ds, int image, int x, int y) {
    /* PixelInstance ctor (random_tree_image.h:140-165) */
    const int aboveValid = (y > 0) ? ds->depth_valid[pix(ds, image, x, y - 1)] : 0;
    const int leftValid = (x > 0) ? ds->depth_valid[pix(ds, image, x - 1, y)] : 0;
    const int aboveLeftValid = (x > 0 && y > 0) ? ds->depth_valid[pix(ds, image, x - 1, y - 1)] : 0;
    const int valid = ds->depth_valid[pix(ds, image, x, y)] - (leftValid + aboveValid - aboveLeftValid);
    if (valid != 1) return std::numeric_limits<float>::quiet_NaN();
    const int64_t above = (y > 0) ? ds->depth_sum[pix(ds, image, x, y - 1)] : 0;
    const int64_t left = (x > 0) ? ds->depth_sum[pix(ds, image, x - 1, y)] : 0;
    const int64_t aboveLeft = (x > 0 && y > 0) ? ds->depth_sum[pix(ds, image, x - 1, y - 1)] : 0;
    const int64_t mm = ds->depth_sum[pix(ds, image, x, y)] - (left + above - aboveLeft);
    if (mm <= 0) return std::numeric_limits<float>::quiet_NaN();
    return static_cast<float>(static_cast<int>(mm)) / 1000.0f; /* Depth::getFloatValue */
}

double orc_feature_response(const orc_dataset* ds, const orc_sample* s, const int8_t* feature11, int flip) {
    return feature_response(ds, s, feature11, flip != 0);
}

void orc_feature_responses(const orc_dataset* ds, int num_samples, const orc_sample* samples, int num_features,
                           const int8_t* features, double* responses) {
    for (int f = 0; f < num_features; f++) {
        int8_t fc[11];
        feature_column(features, num_features, f, fc);
        for (int s = 0; s < num_samples; s++) {
            const bool flip = samples[s].flip == 1;
            responses[static_cast<size_t>(f) * num_samples + s] = feature_response(ds, &samples[s], fc, flip);
        }
    }
}

/* ------------------------------------------------------------------------------------------
 * FeatureEvaluationCPU (random_tree_image.cpp:68-157) and the merge (:339-372)
 * ---------------------------------------------------------------------------------------- */
void orc_histograms(const orc_dataset* ds, int num_samples, const orc_sample* samples, int num_features,
                    int num_thresholds, const int8_t* features, const float* thresholds, int num_classes,
                    uint32_t* counters, int num_threads) {
    const size_t csize = static_cast<size_t>(num_classes) * num_features * num_thresholds * 2;
    std::memset(counters, 0, csize * sizeof(uint32_t));
    std::vector<std::vector<int8_t>> fcols(num_features, std::vector<int8_t>(11));
    std::vector<std::vector<float>> thr(num_features, std::vector<float>(num_thresholds));
    for (int f = 0; f < num_features; f++) {
        feature_column(features, num_features, f, fcols[f].data());
        for (int t = 0; t < num_thresholds; t++) thr[f][t] = thresholds[static_cast<size_t>(t) * num_features + f];
    }
    const size_t labelStride = static_cast<size_t>(num_features) * num_thresholds * 2;
    const size_t featureStride = static_cast<size_t>(num_thresholds) * 2;
    if (num_threads < 1) num_threads = 1;
    /* The reference splits the samples into chunks of max(100, N / numThreads)
     * (random_tree_image.cpp:323) and gives each chunk a private histogram. */
    const int grain = std::max(100, num_samples / num_threads);
    const int num_chunks = (num_samples + grain - 1) / grain;
    std::vector<std::vector<uint32_t>> partial(num_chunks);
#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads)
    for (int chunk = 0; chunk < num_chunks; chunk++) {
        std::vector<uint32_t>& h = partial[chunk];
        h.assign(csize, 0u);
        const int s0 = chunk * grain;
        const int s1 = std::min(num_samples, s0 + grain);
        for (int s = s0; s < s1; s++) {
            const orc_sample* sample = &samples[s];
            const size_t labelOffset = sample->label * labelStride;
            const int setting = sample->flip;
            for (int f = 0; f < num_features; f++) {
                double value1, value2 = 0;
                if (setting == 1) {
                    value1 = feature_response(ds, sample, fcols[f].data(), true);
                } else if (setting == 2) {
                    value1 = feature_response(ds, sample, fcols[f].data(), false);
                    value2 = feature_response(ds, sample, fcols[f].data(), true);
                } else {
                    value1 = feature_response(ds, sample, fcols[f].data(), false);
                }
                const size_t featureOffset = labelOffset + f * featureStride;
                for (int t = 0; t < num_thresholds; t++) {
                    const float threshold = thr[f][t];
                    const int off = static_cast<int>(!(value1 <= threshold));
                    h[featureOffset + t * 2 + off] += 1;
                    if (setting == 2) {
                        const int off2 = static_cast<int>(!(value2 <= threshold));
                        h[featureOffset + t * 2 + off2] += 1;
                    }
                }
            }
        }
    }
    for (int chunk = 0; chunk < num_chunks; chunk++)
        for (size_t i = 0; i < csize; i++) counters[i] += partial[chunk][i];
}

double orc_information_gain(int num_classes, const uint32_t* left, const uint32_t* right, int stride,
                            const uint32_t* all, double total_left, double total_right) {
    /* InformationGainScore::calculateScore (score.h:87-139) */
    const double total = total_left + total_right;
    const double leftProb = total_left / total;
    const double rightProb = total_right / total;
    double score = 0;
    for (int label = 0; label < num_classes; label++) {
        const uint32_t leftValue = left[static_cast<size_t>(label) * stride];
        const uint32_t rightValue = right[static_cast<size_t>(label) * stride];
        const double classProb = all[label] / total;
        if (leftValue > 0) {
            const double classProbLeft = leftValue / total;
            score += classProbLeft * std::log2(classProbLeft / (leftProb * classProb));
        }
        if (rightValue > 0) {
            const double classProbRight = rightValue / total;
            score += classProbRight * std::log2(classProbRight / (rightProb * classProb));
        }
    }
    return normalize_score(score);
}

double orc_score(int num_classes, const uint32_t* left, const uint32_t* right, int stride, const uint32_t* all,
                 double total_left, double total_right) {
    /* NormalizedInformationGainScore::calculateScore (score.h:191-215) */
    const double ig = orc_information_gain(num_classes, left, right, stride, all, total_left, total_right);
    if (ig == 0) return 0;
    const double total = total_left + total_right;
    const double H_s = (entropy(total_left) + entropy(total_right) - entropy(total)) / total;
    double H_c = 0;
    for (int label = 0; label < num_classes; label++) {
        const uint32_t value = all[label];
        if (value > 0) H_c += entropy(value);
    }
    H_c -= entropy(total);
    H_c /= total;
    const double score = (2 * ig) / (H_s + H_c);
    return normalize_score(score);
}

void orc_scores(int num_classes, int num_features, int num_thresholds, const uint32_t* counters,
                const uint32_t* node_histogram, double* scores) {
    /* ImageFeatureEvaluation::calculateScores, host (random_tree_image.cpp:188-237) */
    std::vector<uint32_t> l(num_classes), r(num_classes);
    for (int f = 0; f < num_features; f++) {
        for (int t = 0; t < num_thresholds; t++) {
            double summedLeft = 0, summedRight = 0;
            for (int c = 0; c < num_classes; c++) {
                const size_t idx = ((static_cast<size_t>(c) * num_features + f) * num_thresholds + t) * 2;
                l[c] = counters[idx];
                r[c] = counters[idx + 1];
                summedLeft += l[c];
                summedRight += r[c];
            }
            scores[static_cast<size_t>(t) * num_features + f] =
                orc_score(num_classes, l.data(), r.data(), 1, node_histogram, summedLeft, summedRight);
        }
    }
}

void orc_best_split(int num_features, int num_thresholds, const double* scores, int* best_feature,
                    int* best_threshold, double* best_score) {
    /* random_tree_image.cpp:445-457 */
    double bestScore = -std::numeric_limits<double>::infinity();
    int bestThresh = 0, bestFeat = 0;
    for (int t = 0; t < num_thresholds; t++) {
        for (int f = 0; f < num_features; f++) {
            const double score = scores[static_cast<size_t>(t) * num_features + f];
            if (std::isnan(bestScore) || is_score_better(bestScore, score)) {
                bestFeat = f;
                bestThresh = t;
                bestScore = score;
            }
        }
    }
    *best_feature = bestFeat;
    *best_threshold = bestThresh;
    *best_score = bestScore;
}

/* ------------------------------------------------------------------------------------------
 * Random numbers
 * ---------------------------------------------------------------------------------------- */
void orc_sampler_draws(int seed, int lo, int hi, int count, int32_t* out) {
    Sampler s(seed, lo, hi);
    for (int i = 0; i < count; i++) out[i] = s.next();
}

void orc_philox4x32(uint32_t key0, uint32_t key1, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                    uint32_t* out4) {
    uint32_t c[4] = {c0, c1, c2, c3};
    philox4x32_10(key0, key1, c);
    for (int i = 0; i < 4; i++) out4[i] = c[i];
}

/* generateRandomFeaturesKernel (random_tree_image_gpu.cu:250-390) restated per feature, with
 * the per-feature cuRAND stream replaced by FeatureStream; expressions keep the reference's
 * float operation order (randomOffset :226-238, randomRegion :240-248). */
void orc_generate_features(const orc_dataset* ds, int num_samples, const orc_sample* samples, uint32_t seed,
                           int num_features, int num_thresholds, int box_radius, int region_size,
                           int use_depth_images, int8_t* features, float* thresholds) {
    const int F = num_features;
    std::vector<int8_t> raw(static_cast<size_t>(11) * F);
    std::vector<float> raw_thr(static_cast<size_t>(num_thresholds) * F);
    std::vector<int32_t> keys(F);
    const uint8_t br = static_cast<uint8_t>(static_cast<uint8_t>(box_radius) + 1);
    const uint8_t rs = static_cast<uint8_t>(region_size);
    for (int feat = 0; feat < F; feat++) {
        FeatureStream rng(seed, static_cast<uint32_t>(feat));
        int8_t f[11];
        const uint8_t type = use_depth_images ? static_cast<uint8_t>(feat >= F / 2) : 1;
        f[0] = static_cast<int8_t>(type);
        auto offset = [&](int8_t* vx, int8_t* vy) {
            float t = rng.uniform() * 2.0f;
            t = t * static_cast<float>(br);
            t = t - static_cast<float>(br);
            *vx = static_cast<int8_t>(t);
            float u = rng.uniform() * 2.0f;
            u = u * static_cast<float>(br);
            u = u - static_cast<float>(br);
            *vy = static_cast<int8_t>(u);
        };
        auto region = [&](int8_t* vx, int8_t* vy) {
            float t = rng.uniform() * static_cast<float>(rs);
            t = t + 1.0f;
            *vx = static_cast<int8_t>(t);
            float u = rng.uniform() * static_cast<float>(rs);
            u = u + 1.0f;
            *vy = static_cast<int8_t>(u);
        };
        int8_t o1x, o1y, o2x, o2y, r1x, r1y, r2x, r2y;
        offset(&o1x, &o1y);
        region(&r1x, &r1y);
        /* redraw bounded at 1000 tries, then the x offset moves by one (same rule as the kernel) */
        int redraws = 0;
        do {
            offset(&o2x, &o2y);
            region(&r2x, &r2y);
        } while (o1x == o2x && o1y == o2y && ++redraws < 1000);
        if (o1x == o2x && o1y == o2y) o2x = static_cast<int8_t>(o1x + 1);
        uint8_t ch1 = 0, ch2 = 0;
        if (type == 1) {
            if (use_depth_images) {
                ch1 = static_cast<uint8_t>(feat / (F / 2.0) * 3);
                ch1 %= 3;
                ch2 = static_cast<uint8_t>(feat / (F / 2.0 / 3) * 3);
                ch2 %= 3;
            } else {
                ch1 = static_cast<uint8_t>(feat / (F / 1.0) * 3);
                ch1 %= 3;
                ch2 = static_cast<uint8_t>(feat / (F / 1.0 / 3) * 3);
                ch2 %= 3;
            }
        }
        f[1] = o1x; f[2] = o1y; f[3] = o2x; f[4] = o2y;
        f[5] = r1x; f[6] = r1y; f[7] = r2x; f[8] = r2y;
        f[9] = static_cast<int8_t>(ch1);
        f[10] = static_cast<int8_t>(ch2);
        for (int t = 0; t < num_thresholds; t++) {
            const float scaled = rng.uniform() * static_cast<float>(static_cast<uint32_t>(num_samples - 1));
            const uint32_t idx = static_cast<uint32_t>(scaled);
            double r = feature_response(ds, &samples[idx], f, false);
            if (std::isnan(r)) r = 0.0;
            raw_thr[static_cast<size_t>(t) * F + feat] = static_cast<float>(r);
        }
        for (int r = 0; r < 11; r++) raw[static_cast<size_t>(r) * F + feat] = f[r];
        keys[feat] = sort_key(f);
    }
    /* sortFeatures: order by key; equal keys keep generation order (stable) */
    std::vector<int> order(F);
    for (int i = 0; i < F; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    for (int i = 0; i < F; i++) {
        for (int r = 0; r < 11; r++) features[static_cast<size_t>(r) * F + i] = raw[static_cast<size_t>(r) * F + order[i]];
        for (int t = 0; t < num_thresholds; t++)
            thresholds[static_cast<size_t>(t) * F + i] = raw_thr[static_cast<size_t>(t) * F + order[i]];
    }
}

/* ------------------------------------------------------------------------------------------
 * Breadth-first training (random_tree.h:1249-1415)
 * ---------------------------------------------------------------------------------------- */
int orc_train_tree(const orc_dataset* ds, int num_samples, const orc_sample* samples_in, int num_classes,
                   const orc_train_config* cfg, int* seed_counter, orc_tree_out* out) {
    const int C = num_classes;
    const int F = cfg->num_features, T = cfg->num_thresholds;
    struct Node {
        int index;
        std::vector<orc_sample> samples;
    };
    auto histogram_of = [&](const std::vector<orc_sample>& s, uint32_t* h) {
        /* RandomTree ctor (random_tree.h:507-528): flip Both counts twice */
        for (int c = 0; c < C; c++) h[c] = 0;
        for (const orc_sample& x : s) {
            h[x.label] += 1;
            if (x.flip == 2) h[x.label] += 1;
        }
    };
    auto is_pure = [&](const uint32_t* h) {
        int nz = 0;
        for (int c = 0; c < C; c++)
            if (h[c] != 0) nz++;
        return nz == 1;
    };
    out->num_nodes = 0;
    auto new_node = [&](int level, const std::vector<orc_sample>& s) -> int {
        if (out->num_nodes >= out->max_nodes) return -1;
        const int i = out->num_nodes++;
        out->level[i] = level;
        out->left[i] = -1;
        std::memset(out->feature + static_cast<size_t>(i) * 11, 0, 11);
        out->threshold[i] = std::numeric_limits<float>::quiet_NaN();
        out->score[i] = std::numeric_limits<double>::quiet_NaN();
        out->feature_id[i] = -1;
        histogram_of(s, out->histogram + static_cast<size_t>(i) * C);
        out->num_samples[i] = static_cast<uint32_t>(s.size());
        return i;
    };
    std::vector<orc_sample> root(samples_in, samples_in + num_samples);
    const int rootIndex = new_node(1, root);
    if (rootIndex < 0) return -2;
    std::vector<Node> level_nodes;
    level_nodes.push_back(Node{rootIndex, root});
    int level = 1;
    std::vector<int8_t> features(static_cast<size_t>(11) * F);
    std::vector<float> thresholds(static_cast<size_t>(T) * F);
    std::vector<uint32_t> counters(static_cast<size_t>(C) * F * T * 2);
    std::vector<double> scores(static_cast<size_t>(T) * F);
    while (!level_nodes.empty()) {
        if (level == cfg->max_depth) break;
        /* evaluateBestSplits (random_tree_image.cpp:239-502) */
        std::vector<orc_sample> all;
        for (const Node& n : level_nodes) all.insert(all.end(), n.samples.begin(), n.samples.end());
        Sampler seedSampler = uniform_sampler(seed_counter, 0xFFFFFF);
        const uint32_t seed = static_cast<uint32_t>(seedSampler.next());
        orc_generate_features(ds, static_cast<int>(all.size()), all.data(), seed, F, T, cfg->box_radius,
                              cfg->region_size, cfg->use_depth_images, features.data(), thresholds.data());
        std::vector<Node> next;
        for (Node& node : level_nodes) {
            const uint32_t* hist = out->histogram + static_cast<size_t>(node.index) * C;
            orc_histograms(ds, static_cast<int>(node.samples.size()), node.samples.data(), F, T, features.data(),
                           thresholds.data(), C, counters.data(), cfg->num_threads);
            orc_scores(C, F, T, counters.data(), hist, scores.data());
            int bf, bt;
            double bs;
            orc_best_split(F, T, scores.data(), &bf, &bt, &bs);
            int8_t fcol[11];
            feature_column(features.data(), F, bf, fcol);
            const float threshold = thresholds[static_cast<size_t>(bt) * F + bf];
            /* routing (random_tree.h:1307-1352) */
            std::vector<orc_sample> left, right;
            for (const orc_sample& s0 : node.samples) {
                orc_sample s = s0;
                const int setting = s.flip;
                bool goLeft;
                if (setting == 1) {
                    goLeft = feature_response(ds, &s, fcol, true) <= threshold;
                } else {
                    goLeft = feature_response(ds, &s, fcol, false) <= threshold;
                }
                bool same = true;
                if (setting == 2) same = (feature_response(ds, &s, fcol, true) <= threshold) == goLeft;
                if (setting == 2 && !same) s.flip = 0;
                if (goLeft) {
                    left.push_back(s);
                    if (setting == 2 && !same) {
                        orc_sample copy = s0;
                        copy.flip = 1;
                        right.push_back(copy);
                    }
                } else {
                    right.push_back(s);
                    if (setting == 2 && !same) {
                        orc_sample copy = s0;
                        copy.flip = 1;
                        left.push_back(copy);
                    }
                }
            }
            if (left.empty() || right.empty()) return -1;
            const int li = new_node(level + 1, left);
            const int ri = new_node(level + 1, right);
            if (li < 0 || ri < 0) return -2;
            out->left[node.index] = li;
            std::memcpy(out->feature + static_cast<size_t>(node.index) * 11, fcol, 11);
            out->threshold[node.index] = threshold;
            out->score[node.index] = bs;
            out->feature_id[node.index] = bf;
            const uint32_t* lh = out->histogram + static_cast<size_t>(li) * C;
            const uint32_t* rh = out->histogram + static_cast<size_t>(ri) * C;
            /* shouldContinueGrowing (random_tree.h:1182-1191) */
            if (!is_pure(lh) && left.size() >= static_cast<size_t>(cfg->min_sample_count))
                next.push_back(Node{li, std::move(left)});
            if (!is_pure(rh) && right.size() >= static_cast<size_t>(cfg->min_sample_count))
                next.push_back(Node{ri, std::move(right)});
        }
        level_nodes.swap(next);
        level++;
    }
    return 0;
}

void orc_normalize_histogram(int num_classes, const uint32_t* histogram, const uint32_t* prior,
                             double histogram_bias, int use_labels_prior, double* out) {
    /* detail::normalizeHistogram (random_tree.cpp:54-104) */
    std::vector<double> labelWeights(num_classes);
    double psum = 0;
    for (int i = 0; i < num_classes; i++) psum += prior[i];
    for (int i = 0; i < num_classes; i++) labelWeights[i] = prior[i] / psum;
    double sum = 0;
    for (int i = 0; i < num_classes; i++) sum += histogram[i];
    for (int i = 0; i < num_classes; i++) {
        out[i] = histogram[i] - histogram_bias * sum;
        if (out[i] < 0.0) out[i] = 0.0;
    }
    sum = 0;
    for (int i = 0; i < num_classes; i++) sum += out[i];
    if (sum > 0) {
        for (int i = 0; i < num_classes; i++) {
            if (use_labels_prior)
                out[i] = out[i] / sum * labelWeights[i];
            else
                out[i] = out[i] / sum;
        }
    }
}

/* ------------------------------------------------------------------------------------------
 * CPU prediction (random_forest_image.cpp:307-345; random_tree.h:613-622, 989-1002)
 * ---------------------------------------------------------------------------------------- */
void orc_predict(const orc_dataset* ds, int image, int num_trees, const orc_tree_view* trees, int num_classes,
                 float* probabilities, uint8_t* labels, int num_threads) {
    const int W = ds->width, H = ds->height, C = num_classes;
    const size_t hw = static_cast<size_t>(W) * H;
    if (num_threads < 1) num_threads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads)
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            const size_t p = static_cast<size_t>(y) * W + x;
            for (int c = 0; c < C; c++) probabilities[c * hw + p] = 0.0f;
            orc_sample px;
            px.x = static_cast<uint16_t>(x);
            px.y = static_cast<uint16_t>(y);
            px.image = static_cast<uint32_t>(image);
            const float d = orc_pixel_depth(ds, image, x, y);
            px.depth = std::isnan(d) ? 0.0f : d;
            px.label = 0;
            px.flip = 0;
            px.reserved = 0;
            for (int t = 0; t < num_trees; t++) {
                const orc_tree_view& tree = trees[t];
                int node = 0;
                while (tree.left[node] >= 0) {
                    const double r = feature_response(ds, &px, tree.feature + static_cast<size_t>(node) * 11, false);
                    node = (r <= tree.threshold[node]) ? tree.left[node] : tree.left[node] + 1;
                }
                const double* hist = tree.normalized + static_cast<size_t>(node) * C;
                for (int c = 0; c < C; c++) {
                    float& v = probabilities[c * hw + p];
                    v = static_cast<float>(v + hist[c]);
                }
            }
            double sum = 0.0;
            for (int c = 0; c < C; c++) sum += probabilities[c * hw + p];
            float bestProb = -1.0f;
            uint8_t label = 0;
            for (int c = 0; c < C; c++) {
                float& v = probabilities[c * hw + p];
                v = static_cast<float>(v / sum);
                const float prob = v;
                if (prob > bestProb) {
                    label = static_cast<uint8_t>(c);
                    bestProb = prob;
                }
            }
            labels[p] = label;
        }
    }
}

/* ------------------------------------------------------------------------------------------
 * Class-uniform sampling (random_tree_image.cpp:911-1059) and the block sort (:776-802)
 * ---------------------------------------------------------------------------------------- */
int orc_sample_class_uniform(int n, int width, int height, const uint8_t* labels, const uint16_t* depth_mm,
                             int num_classes, const uint8_t* ignore, int subsample_count, int* seed_counter,
                             int capacity, orc_sample* out) {
    int numLabels = num_classes;
    for (int c = 0; c < num_classes; c++)
        if (ignore[c]) numLabels--;
    const size_t samplesPerClass =
        static_cast<size_t>(std::ceil(n * static_cast<double>(subsample_count) / static_cast<double>(numLabels)));
    Sampler seedSampler = uniform_sampler(seed_counter, 0xFFFFFF);
    const int randomSeed = seedSampler.next();
    struct Reservoir {
        size_t count = 0;
        std::vector<orc_sample> items;
    };
    std::vector<Reservoir> res(num_classes);
    int chunkSeed = randomSeed;
    Sampler sampler = uniform_sampler(&chunkSeed, 0x7FFFFFFF);
    const size_t hw = static_cast<size_t>(width) * height;
    for (int img = 0; img < n; img++) {
        for (int y = 0; y < height; y++) {
            for (int x = 0; x < width; x++) {
                const size_t p = img * hw + static_cast<size_t>(y) * width + x;
                const uint8_t label = labels[p];
                if (ignore[label]) continue;
                const uint16_t d = depth_mm[p];
                if (d == 0) continue;
                orc_sample s;
                s.x = static_cast<uint16_t>(x);
                s.y = static_cast<uint16_t>(y);
                s.image = static_cast<uint32_t>(img);
                s.depth = static_cast<float>(static_cast<int>(d)) / 1000.0f;
                s.label = label;
                s.flip = 0;
                s.reserved = 0;
                Reservoir& r = res[label];
                /* ReservoirSampler::sample (random_tree.h:1085-1105) */
                if (r.items.size() < samplesPerClass) {
                    r.items.push_back(s);
                } else {
                    const size_t rnd = static_cast<size_t>(sampler.next()) % (r.count + 1);
                    if (rnd < samplesPerClass) r.items[rnd] = s;
                }
                r.count++;
            }
        }
    }
    /* merge sampler takes one more seed; with a single chunk it draws nothing */
    (void)uniform_sampler(seed_counter, 0x7FFFFFFF);
    std::vector<orc_sample> all;
    for (int label = 0; label < num_classes; label++) {
        if (ignore[label]) continue;
        /* allSubsamples.insert(begin, ...) prepends each class */
        all.insert(all.begin(), res[label].items.begin(), res[label].items.end());
    }
    if (all.size() != samplesPerClass * numLabels) return -1;
    const size_t block = 200000;
    for (size_t b = 0; b < all.size(); b += block) {
        const size_t e = std::min(all.size(), b + block);
        std::stable_sort(all.begin() + b, all.begin() + e, [](const orc_sample& a, const orc_sample& c) {
            if (a.image != c.image) return a.image < c.image;
            if (a.label != c.label) return a.label < c.label;
            if (a.y / 10 != c.y / 10) return a.y / 10 < c.y / 10;
            if (a.x / 10 != c.x / 10) return a.x / 10 < c.x / 10;
            return false;
        });
    }
    if (static_cast<int>(all.size()) > capacity) return -2;
    std::copy(all.begin(), all.end(), out);
    return static_cast<int>(all.size());
}

/* Pixel-uniform sampling (random_tree_image.cpp:840-883): the image of each sample from one Sampler
 * over the image list, its pixel from two fresh Samplers of the random source (x, then y), redrawn
 * together while the label is ignored; then the block sort as above. Returns the count. */
int orc_sample_pixel_uniform(int n, int width, int height, const uint8_t* labels, const uint16_t* depth_mm,
                             const uint8_t* ignore, int subsample_count, int* seed_counter, int capacity,
                             orc_sample* out) {
    Sampler rgen_image = uniform_sampler(seed_counter, n);
    const size_t hw = static_cast<size_t>(width) * height;
    std::vector<orc_sample> all;
    for (size_t k = 0; k < static_cast<size_t>(subsample_count) * n; k++) {
        const int img = rgen_image.next();
        Sampler rgen_x = uniform_sampler(seed_counter, width);
        Sampler rgen_y = uniform_sampler(seed_counter, height);
        for (long long tries = 0;; tries++) {
            if (tries >= 100000000LL) return -1;
            const int x = rgen_x.next(), y = rgen_y.next();
            const size_t p = img * hw + static_cast<size_t>(y) * width + x;
            if (ignore[labels[p]]) continue;
            orc_sample s;
            s.x = static_cast<uint16_t>(x);
            s.y = static_cast<uint16_t>(y);
            s.image = static_cast<uint32_t>(img);
            const uint16_t d = depth_mm[p];
            s.depth = d > 0 ? static_cast<float>(static_cast<int>(d)) / 1000.0f : 0.0f;
            s.label = labels[p];
            s.flip = 0;
            s.reserved = 0;
            all.push_back(s);
            break;
        }
    }
    const size_t block = 200000;
    for (size_t b = 0; b < all.size(); b += block) {
        const size_t e = std::min(all.size(), b + block);
        std::stable_sort(all.begin() + b, all.begin() + e, [](const orc_sample& a, const orc_sample& c) {
            if (a.image != c.image) return a.image < c.image;
            if (a.label != c.label) return a.label < c.label;
            if (a.y / 10 != c.y / 10) return a.y / 10 < c.y / 10;
            if (a.x / 10 != c.x / 10) return a.x / 10 < c.x / 10;
            return false;
        });
    }
    if (static_cast<int>(all.size()) > capacity) return -2;
    std::copy(all.begin(), all.end(), out);
    return static_cast<int>(all.size());
}

/* RGBDImage::fillDepth (image.cpp:279-377): passes from the right, left, top and bottom, each
 * replacing a 0 by its already-processed neighbour. depth uint16 [n][H][W], in place. */
void orc_fill_depth(int n, int width, int height, uint16_t* depth) {
    for (int i = 0; i < n; i++) {
        uint16_t* d = depth + static_cast<size_t>(i) * width * height;
        for (int y = 0; y < height; y++)
            for (int x = width - 2; x >= 0; x--)
                if (!d[y * width + x]) d[y * width + x] = d[y * width + x + 1];
        for (int y = 0; y < height; y++)
            for (int x = 1; x < width; x++)
                if (!d[y * width + x]) d[y * width + x] = d[y * width + x - 1];
        for (int y = 1; y < height; y++)
            for (int x = 0; x < width; x++)
                if (!d[y * width + x]) d[y * width + x] = d[(y - 1) * width + x];
        for (int y = height - 2; y >= 0; y--)
            for (int x = 0; x < width; x++)
                if (!d[y * width + x]) d[y * width + x] = d[(y + 1) * width + x];
    }
}

/* CIE 1976 L*a*b* of linear RGB / 255 (BT.709 primaries, D65 white), rounded to float:
 * rgb uint8 [n][H][W][3] -> lab float [n][3][H][W]. */
static double lab_f(double t) {
    return t > 216.0 / 24389.0 ? std::cbrt(t) : t * (841.0 / 108.0) + 4.0 / 29.0;
}

void orc_rgb_to_lab(int n, int width, int height, const uint8_t* rgb, float* lab) {
    const size_t plane = static_cast<size_t>(width) * height;
    for (size_t i = 0; i < n * plane; i++) {
        const double r = rgb[3 * i] / 255.0, g = rgb[3 * i + 1] / 255.0, b = rgb[3 * i + 2] / 255.0;
        const double X = 0.412453 * r + 0.357580 * g + 0.180423 * b;
        const double Y = 0.212671 * r + 0.715160 * g + 0.072169 * b;
        const double Z = 0.019334 * r + 0.119193 * g + 0.950227 * b;
        const double fx = lab_f(X / 0.950456), fy = lab_f(Y), fz = lab_f(Z / 1.088754);
        const size_t img = i / plane, p = i % plane;
        float* out = lab + img * 3 * plane + p;
        out[0] = static_cast<float>(116.0 * fy - 16.0);
        out[plane] = static_cast<float>(500.0 * (fx - fy));
        out[2 * plane] = static_cast<float>(200.0 * (fy - fz));
    }
}

/* Mean softmax cross-entropy of the refinement network and its gradient, in double (the CPU
 * reference for curfil_b200's training kernels). params float: W1 [H][D], b1 [H], W2 [C][H], b2 [C]. */
void orc_mlp_loss_grad(int n, int D, int H, int C, const float* params, const float* X, const uint8_t* Y,
                       double* grad, double* loss) {
    const float* W1 = params;
    const float* b1 = W1 + static_cast<size_t>(H) * D;
    const float* W2 = b1 + H;
    const float* b2 = W2 + static_cast<size_t>(C) * H;
    const size_t P = static_cast<size_t>(H) * D + H + static_cast<size_t>(C) * H + C;
    std::fill(grad, grad + P, 0.0);
    double* gW1 = grad;
    double* gb1 = gW1 + static_cast<size_t>(H) * D;
    double* gW2 = gb1 + H;
    double* gb2 = gW2 + static_cast<size_t>(C) * H;
    double total = 0;
    std::vector<double> h(H), z(C), dz(C), g(H);
    for (int r = 0; r < n; r++) {
        const float* x = X + static_cast<size_t>(r) * D;
        for (int j = 0; j < H; j++) {
            double a = b1[j];
            for (int k = 0; k < D; k++) a += static_cast<double>(W1[static_cast<size_t>(j) * D + k]) * x[k];
            h[j] = a > 0 ? a : 0;
        }
        double m = -std::numeric_limits<double>::infinity();
        for (int c = 0; c < C; c++) {
            double a = b2[c];
            for (int j = 0; j < H; j++) a += static_cast<double>(W2[static_cast<size_t>(c) * H + j]) * h[j];
            z[c] = a;
            m = std::max(m, a);
        }
        double s = 0;
        for (int c = 0; c < C; c++) s += std::exp(z[c] - m);
        total += std::log(s) + m - z[Y[r]];
        for (int c = 0; c < C; c++) dz[c] = (std::exp(z[c] - m) / s - (c == Y[r] ? 1.0 : 0.0)) / n;
        for (int j = 0; j < H; j++) {
            double a = 0;
            for (int c = 0; c < C; c++) a += static_cast<double>(W2[static_cast<size_t>(c) * H + j]) * dz[c];
            g[j] = h[j] > 0 ? a : 0;
        }
        for (int c = 0; c < C; c++) {
            gb2[c] += dz[c];
            for (int j = 0; j < H; j++) gW2[static_cast<size_t>(c) * H + j] += dz[c] * h[j];
        }
        for (int j = 0; j < H; j++) {
            gb1[j] += g[j];
            for (int k = 0; k < D; k++) gW1[static_cast<size_t>(j) * D + k] += g[j] * x[k];
        }
    }
    *loss = total / n;
}

/* The device classUniform sampler's definition (curfil_b200 cf_sample_tree_pixels_device): keys
 * from Philox4x32-10 per eligible pixel, the per-class quota of smallest (key, pixel index), order
 * (image, label, y/10, x/10, y, x). Same seed draws as the reservoir sampler above. */
int orc_sample_class_uniform_keys(int n, int width, int height, const uint8_t* labels, const uint16_t* depth_mm,
                                  int num_classes, const uint8_t* ignore, int subsample_count, int* seed_counter,
                                  int capacity, orc_sample* out) {
    int numLabels = num_classes;
    for (int c = 0; c < num_classes; c++)
        if (ignore[c]) numLabels--;
    const size_t samplesPerClass =
        static_cast<size_t>(std::ceil(n * static_cast<double>(subsample_count) / static_cast<double>(numLabels)));
    Sampler seedSampler = uniform_sampler(seed_counter, 0xFFFFFF);
    const uint32_t k0 = static_cast<uint32_t>(seedSampler.next());
    (void)uniform_sampler(seed_counter, 0x7FFFFFFF);
    const size_t hw = static_cast<size_t>(width) * height;
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> keys(num_classes);   // (key, pixel index)
    for (size_t i = 0; i < n * hw; i++) {
        const uint8_t label = labels[i];
        if (label >= num_classes || ignore[label] || depth_mm[i] == 0) continue;
        uint32_t c[4] = {static_cast<uint32_t>(i), 0u, 0u, 0u};
        philox4x32_10(k0, 0x53414D50u, c);
        keys[label].emplace_back(c[0], static_cast<uint32_t>(i));
    }
    std::vector<orc_sample> all;
    for (int label = 0; label < num_classes; label++) {
        if (ignore[label]) continue;
        auto& v = keys[label];
        if (v.size() < samplesPerClass) return -1;
        std::sort(v.begin(), v.end());
        for (size_t j = 0; j < samplesPerClass; j++) {
            const size_t i = v[j].second;
            const size_t img = i / hw, p = i % hw;
            orc_sample s;
            s.x = static_cast<uint16_t>(p % width);
            s.y = static_cast<uint16_t>(p / width);
            s.image = static_cast<uint32_t>(img);
            s.depth = static_cast<float>(static_cast<int>(depth_mm[i])) / 1000.0f;
            s.label = static_cast<uint8_t>(label);
            s.flip = 0;
            s.reserved = 0;
            all.push_back(s);
        }
    }
    std::sort(all.begin(), all.end(), [](const orc_sample& a, const orc_sample& b) {
        if (a.image != b.image) return a.image < b.image;
        if (a.label != b.label) return a.label < b.label;
        if (a.y / 10 != b.y / 10) return a.y / 10 < b.y / 10;
        if (a.x / 10 != b.x / 10) return a.x / 10 < b.x / 10;
        if (a.y != b.y) return a.y < b.y;
        return a.x < b.x;
    });
    if (static_cast<int>(all.size()) > capacity) return -2;
    std::copy(all.begin(), all.end(), out);
    return static_cast<int>(all.size());
}

}  // extern "C"

/* ------------------------------------------------------------------------------------------
 * Synthetic frames (the workloads' data, see oracle.h)
 * ---------------------------------------------------------------------------------------- */
namespace {

/* SplitMix64 stream; uniform doubles from its top 53 bits, normals by Box-Muller. */
class Mix64 {
public:
    explicit Mix64(uint64_t s) : state_(s) {}
    uint64_t bits() {
        state_ += 0x9E3779B97F4A7C15ull;
        uint64_t z = state_;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double unit() { return static_cast<double>(bits() >> 11) * (1.0 / 9007199254740992.0); }
    int index(int n) { return static_cast<int>(unit() * n); }
    double gauss() {
        const double a = std::max(unit(), 1e-300);
        const double b = unit();
        return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
    }

private:
    uint64_t state_;
};

struct Cell {
    double x, y, r, g, b, depth, slope_x, slope_y;
    int cls;
};

void synthetic_frame(uint64_t seed, int frame, int W, int H, int K, int C, const double* class_rgb,
                     const double* class_depth, uint8_t* rgb, uint16_t* depth, uint8_t* labels) {
    Mix64 rng(seed * 0x100000001B3ull + static_cast<uint64_t>(frame) * 0x9E3779B97F4A7C15ull + 17);
    std::vector<Cell> cells(K);
    for (Cell& c : cells) {
        c.x = rng.unit() * W;
        c.y = rng.unit() * H;
        c.cls = rng.index(C);
        c.r = class_rgb[3 * c.cls + 0] + (rng.unit() - 0.5) * 30.0;
        c.g = class_rgb[3 * c.cls + 1] + (rng.unit() - 0.5) * 30.0;
        c.b = class_rgb[3 * c.cls + 2] + (rng.unit() - 0.5) * 30.0;
        c.depth = class_depth[c.cls] + (rng.unit() - 0.5) * 600.0;
        c.slope_x = (rng.unit() - 0.5) * 4.0;
        c.slope_y = (rng.unit() - 0.5) * 4.0;
    }
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            const Cell* near = &cells[0];
            double best = 1e300;
            for (const Cell& c : cells) {
                const double d2 = (x - c.x) * (x - c.x) + (y - c.y) * (y - c.y);
                if (d2 < best) {
                    best = d2;
                    near = &c;
                }
            }
            const size_t p = static_cast<size_t>(y) * W + x;
            const double base[3] = {near->r, near->g, near->b};
            for (int k = 0; k < 3; k++) {
                const double v = std::round(base[k] + 8.0 * rng.gauss());
                rgb[3 * p + k] = static_cast<uint8_t>(std::min(255.0, std::max(0.0, v)));
            }
            const double plane = near->depth + near->slope_x * (x - near->x) + near->slope_y * (y - near->y);
            const double clamped = std::min(5000.0, std::max(500.0, plane));
            depth[p] = rng.unit() < 0.1 ? 0 : static_cast<uint16_t>(std::lround(clamped));
            int label = near->cls;
            if (C > 1 && rng.unit() < 0.05) {
                const int other = rng.index(C - 1);
                label = other >= label ? other + 1 : other;
            }
            labels[p] = static_cast<uint8_t>(label);
        }
    }
}

}  // namespace

extern "C" void orc_synthetic_frames(uint64_t seed, int first, int n, int width, int height, int num_cells,
                                     int num_classes, uint8_t* rgb, uint16_t* depth_mm, uint8_t* labels) {
    Mix64 crng(seed ^ 0xC1A55E5ull);
    std::vector<double> class_rgb(3 * num_classes), class_depth(num_classes);
    for (int c = 0; c < num_classes; c++) {
        for (int k = 0; k < 3; k++) class_rgb[3 * c + k] = 30.0 + 195.0 * crng.unit();
        class_depth[c] = 900.0 + 3600.0 * crng.unit();
    }
    const size_t plane = static_cast<size_t>(width) * height;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; i++)
        synthetic_frame(seed, first + i, width, height, num_cells, num_classes, class_rgb.data(), class_depth.data(),
                        rgb + 3 * plane * i, depth_mm + plane * i, labels + plane * i);
}
