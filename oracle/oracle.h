/*
 * CPU oracle for the CURFIL training split search and dense prediction path.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates, in plain C++, what the reference
 * (deeplearningais/curfil) computes on its CPU path, so that the CUDA implementation in
 * curfil_b200/ can be checked against it. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load it; the product never does.
 *
 * Every function cites the reference file:line it follows (paths relative to the
 * reference project root).  Parity is pinned against the known-answer values of the
 * reference's own unit tests (tests/golden/reference_kats.py); the random-number streams
 * (Boost.Random, cuRAND) cannot be pinned, see the notes on each generator.
 */
#ifndef CURFIL_ORACLE_H
#define CURFIL_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One pixel sample; same 16-byte layout as cf_sample in include/curfil_b200.h.
 * Mirrors PixelInstance (src/curfil/random_tree_image.h:140-181) with the image pointer
 * replaced by an index into the dataset. */
typedef struct orc_sample {
    uint16_t x, y;
    uint32_t image;
    float depth;      /* metres, Depth::getFloatValue() = mm / 1000.0f (image.h:146-149) */
    uint8_t label;
    uint8_t flip;     /* HorizontalFlipSetting: 0 NoFlip, 1 Flip, 2 Both (random_tree.h:58-60) */
    uint16_t reserved;
} orc_sample;

/* Integral images of n images of equal size, in the reference layout
 * (image.h:420-421): colour float[n][3][H][W]; depth sum and valid count [n][H][W].
 * The depth sum is held in int64 here: the reference's int overflows for 1280x960
 * frames (image.cpp:270-274), box differences are exact in int64. */
typedef struct orc_dataset {
    int n, width, height;
    const float* color;
    const int64_t* depth_sum;
    const int32_t* depth_valid;
} orc_dataset;

/* --- integral images ------------------------------------------------------------------ */
/* RGBDImage::calculateIntegral (image.cpp:236-277, 531-556): row-major scan in double with
 * one Kahan carry across the image, stored to float (colour) / int (depth). rgb is the
 * interleaved raw frame [H][W][3] (uint8), depth_mm [H][W] (0 = missing). */
void orc_integral(int width, int height, const uint8_t* rgb, const uint16_t* depth_mm,
                  float* color_out, int64_t* depth_sum_out, int32_t* depth_valid_out);

/* Same scan for an arbitrary float colour plane set [3][H][W] (used by the KATs that set
 * non-integer colours, random_tree_image_gpu_test.cu:700-715). */
void orc_integral_float_color(int width, int height, const float* color_in, float* color_out);

/* Pixel depth recovered from the integral image (random_tree_image.h:140-165).
 * Returns the depth in metres or NaN when the pixel has no valid depth. */
float orc_pixel_depth(const orc_dataset* ds, int image, int x, int y);

/* --- feature responses ------------------------------------------------------------------ */
/* ImageFeatureFunction::calculateFeatureResponse (random_tree_image.h:485-623).
 * feature points at the 11 int8 parameters in ImageFeaturesAndThresholds row order
 * (type, o1x, o1y, o2x, o2y, r1x, r1y, r2x, r2y, ch1, ch2; random_tree_image.h:686-759). */
double orc_feature_response(const orc_dataset* ds, const orc_sample* s, const int8_t* feature11,
                            int flip_region);

/* responses[f][s] for features given as int8[11][F] (column f = feature f). */
void orc_feature_responses(const orc_dataset* ds, int num_samples, const orc_sample* samples,
                           int num_features, const int8_t* features, double* responses);

/* --- split search ----------------------------------------------------------------------- */
/* FeatureEvaluationCPU (random_tree_image.cpp:68-157) + merge (:339-372): counters
 * uint32[C][F][T][2] (index 0 = left, 1 = right), per-thread private histograms. */
void orc_histograms(const orc_dataset* ds, int num_samples, const orc_sample* samples,
                    int num_features, int num_thresholds, const int8_t* features,
                    const float* thresholds, int num_classes, uint32_t* counters, int num_threads);

/* NormalizedInformationGainScore::calculateScore (score.h:87-215) */
double orc_score(int num_classes, const uint32_t* left, const uint32_t* right, int stride,
                 const uint32_t* all, double total_left, double total_right);
/* InformationGainScore::calculateScore (score.h:87-139) */
double orc_information_gain(int num_classes, const uint32_t* left, const uint32_t* right, int stride,
                            const uint32_t* all, double total_left, double total_right);

/* ImageFeatureEvaluation::calculateScores (random_tree_image.cpp:188-237): scores[T][F]. */
void orc_scores(int num_classes, int num_features, int num_thresholds, const uint32_t* counters,
                const uint32_t* node_histogram, double* scores);

/* Thresh-major, feature-minor argmax with detail::isScoreBetter
 * (random_tree_image.cpp:445-457, random_tree.cpp:36-52). */
void orc_best_split(int num_features, int num_thresholds, const double* scores,
                    int* best_feature, int* best_threshold, double* best_score);

/* --- random numbers ---------------------------------------------------------------------- */
/* Sampler(seed, lo, hi).getNext() draws (random_tree.h:1009-1063): mt19937 seeded with
 * `seed`, uniform integer on [lo, hi] with the bucket-rejection method of Boost.Random's
 * uniform_int (Boost >= 1.47; the reference pins no Boost version, so unpinned).
 * Writes `count` consecutive draws. */
void orc_sampler_draws(int seed, int lo, int hi, int count, int32_t* out);

/* GPU-style candidate generation (random_tree_image_gpu.cu:250-390 structure; the cuRAND
 * XORWOW stream is replaced by Philox4x32-10, Salmon et al. SC'11) followed by the stable
 * sort by getSortKey (random_tree_image.h:444-452, random_tree_image.cpp:504-566).
 * features int8[11][F], thresholds float[T][F]. */
void orc_generate_features(const orc_dataset* ds, int num_samples, const orc_sample* samples,
                           uint32_t seed, int num_features, int num_thresholds, int box_radius,
                           int region_size, int use_depth_images, int8_t* features,
                           float* thresholds);
/* Philox4x32-10 block for (key, counter) -> 4 words. Exposed for the RNG unit test. */
void orc_philox4x32(uint32_t key0, uint32_t key1, uint32_t c0, uint32_t c1, uint32_t c2,
                    uint32_t c3, uint32_t* out4);

/* --- training ---------------------------------------------------------------------------- */
typedef struct orc_train_config {
    int num_features;       /* featureCount */
    int num_thresholds;     /* thresholds */
    int max_depth;          /* maxDepth (root is level 1) */
    int min_sample_count;   /* minSampleCount */
    int box_radius;         /* offset range */
    int region_size;        /* box half-size range */
    int use_depth_images;
    int num_threads;        /* host threads for the histogram loop */
} orc_train_config;

/* Output of a trained tree, nodes in breadth-first id order (index = nodeId - treeId).
 * Arrays are allocated by the caller with capacity `max_nodes`. */
typedef struct orc_tree_out {
    int max_nodes;
    int num_nodes;           /* written */
    int32_t* level;          /* [max_nodes] */
    int32_t* left;           /* [max_nodes] index of left child, -1 for leaves; right = left + 1 */
    int8_t* feature;         /* [max_nodes][11] split parameters */
    float* threshold;        /* [max_nodes] */
    double* score;           /* [max_nodes] */
    int32_t* feature_id;     /* [max_nodes] index of the feature in its level's sorted table */
    uint32_t* histogram;     /* [max_nodes][C] */
    uint32_t* num_samples;   /* [max_nodes] */
} orc_tree_out;

/* RandomTreeTrain::train (random_tree.h:1249-1415) driving evaluateBestSplits
 * (random_tree_image.cpp:239-502) with CPU evaluation and GPU-style candidate generation
 * (one table per level, seed drawn from the tree's RandomSource at seed counter
 * *seed_counter, which is advanced). Returns 0, or a negative code: -1 empty child
 * ("no samples in left/right node", random_tree.h:1388-1393), -2 capacity exceeded. */
int orc_train_tree(const orc_dataset* ds, int num_samples, const orc_sample* samples,
                   int num_classes, const orc_train_config* cfg, int* seed_counter,
                   orc_tree_out* out);

/* detail::normalizeHistogram (random_tree.cpp:54-104). */
void orc_normalize_histogram(int num_classes, const uint32_t* histogram, const uint32_t* prior,
                             double histogram_bias, int use_labels_prior, double* out);

/* RandomForestImage::predict CPU branch (random_forest_image.cpp:307-345): trees are given
 * by their node arrays (left, feature, threshold) and per-node normalised histograms
 * (double [nodes][C]). probabilities float[C][H][W], labels uint8[H][W]. */
typedef struct orc_tree_view {
    int num_nodes;
    const int32_t* left;
    const int8_t* feature;
    const float* threshold;
    const double* normalized;    /* [num_nodes][C] */
} orc_tree_view;

void orc_predict(const orc_dataset* ds, int image, int num_trees, const orc_tree_view* trees,
                 int num_classes, float* probabilities, uint8_t* labels, int num_threads);

/* --- sampling ---------------------------------------------------------------------------- */
/* RandomTreeImage::subsampleTrainingDataClassUniform (random_tree_image.cpp:911-1059) with
 * one host thread (the reference is nondeterministic with more), followed by the block sort
 * by (image, label, y/10, x/10) of RandomTreeImage::train (random_tree_image.cpp:776-802),
 * done with a stable sort. labels uint8[n][H][W]; ignore[C] marks ignored classes.
 * Returns the number of samples written (<= capacity), or -1 when the reference would throw
 * "failed to sample enough pixels". */
int orc_sample_class_uniform(int n, int width, int height, const uint8_t* labels,
                             const uint16_t* depth_mm, int num_classes, const uint8_t* ignore,
                             int subsample_count, int* seed_counter, int capacity,
                             orc_sample* out);
/* Pixel-uniform sampling (random_tree_image.cpp:840-883) with the block sort; returns the count. */
int orc_sample_pixel_uniform(int n, int width, int height, const uint8_t* labels, const uint16_t* depth_mm,
                             const uint8_t* ignore, int subsample_count, int* seed_counter, int capacity,
                             orc_sample* out);
/* RGBDImage::fillDepth (image.cpp:279-377) on depth uint16 [n][H][W], in place. */
void orc_fill_depth(int n, int width, int height, uint16_t* depth);
/* CIE 1976 L*a*b* (linear RGB / 255, BT.709 primaries, D65 white; the published formulas the
 * reference's Vigra RGB2LabFunctor implements), rounded to float: lab [n][3][H][W]. */
void orc_rgb_to_lab(int n, int width, int height, const uint8_t* rgb, float* lab);

/* Mean softmax cross-entropy of the project's per-pixel refinement network (h = relu(W1 x + b1),
 * z = W2 h + b2) over n rows X [n][D] with labels Y [n], and its gradient [P], in double. Not a
 * reference algorithm: the CPU check of the network's training kernels. */
void orc_mlp_loss_grad(int n, int D, int H, int C, const float* params, const float* X, const uint8_t* Y,
                       double* grad, double* loss);

/* The definition of the project's device classUniform sampler (not a reference algorithm): every
 * eligible pixel i (label not ignored, depth > 0; i = image * H * W + y * W + x) gets the key
 * Philox4x32-10(key = (s, 0x53414D50), counter = (i, 0, 0, 0)) word 0, s = the reference
 * sampler's randomSeed draw; each class keeps its quota of smallest (key, i); samples ordered by
 * (image, label, y/10, x/10, y, x). Returns the count, -1 if a class has too few pixels. */
int orc_sample_class_uniform_keys(int n, int width, int height, const uint8_t* labels,
                                  const uint16_t* depth_mm, int num_classes, const uint8_t* ignore,
                                  int subsample_count, int* seed_counter, int capacity,
                                  orc_sample* out);

/* The seeded synthetic RGB-D frames every workload here is made of (not a reference algorithm: the
 * stand-in for recorded data). Per frame, from (seed, frame index): a Voronoi partition into
 * num_cells cells, each taking a class with a class colour and depth shared by all frames; colour
 * uint8 RGB = cell colour + N(0, 8^2) noise; depth uint16 mm = a plane per cell clamped to
 * [500, 5000], 10% of pixels 0; labels = cell class with 5% flipped to another class. Frames
 * first .. first + n - 1: rgb [n][H][W][3], depth [n][H][W], labels [n][H][W]. Restated here so that
 * the CPU baseline needs nothing from the product library; a test pins it to the library's
 * generator byte for byte. */
void orc_synthetic_frames(uint64_t seed, int first, int n, int width, int height, int num_cells,
                          int num_classes, uint8_t* rgb, uint16_t* depth_mm, uint8_t* labels);

#ifdef __cplusplus
}
#endif

#endif
