/*
 * curfil_b200 C-ABI: the drop-in boundary for CURFIL's random-forest training split search and
 * dense per-pixel prediction, implemented with hand-written sm_100a CUDA kernels.
 *
 * Plain pointers and sizes only; every entry point returns a cf_status and records a message
 * retrievable with cf_last_error(). Host buffers are owned by the caller. Device memory is owned
 * by the objects (context, dataset, forest, server) that allocate it, except where a function
 * says it takes device pointers. Each declaration names the reference interface it replaces
 * (paths relative to the deeplearningais/curfil project root).
 */
#ifndef CURFIL_B200_H
#define CURFIL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t cf_status;
#define CF_OK 0
#define CF_ERR_INVALID 1       /* bad argument or configuration (reference: std::runtime_error) */
#define CF_ERR_CUDA 2          /* CUDA runtime error (reference: cudaSafeCall, utils.h:48) */
#define CF_ERR_OOM 3           /* device allocation failed */
#define CF_ERR_EMPTY_CHILD 4   /* "no samples in left/right node" (random_tree.h:1388-1393) */
#define CF_ERR_CAPACITY 5      /* a fixed capacity was exceeded */
#define CF_ERR_TIMEOUT 6       /* a bounded wait ran out */
#define CF_ERR_REJECTED 7      /* serving admission refused the request */
#define CF_ERR_IO 8            /* file read/write or format error */
#define CF_ERR_STATE 9         /* object used in the wrong state */

typedef struct cf_context cf_context;
typedef struct cf_dataset cf_dataset;
typedef struct cf_tree cf_tree;
typedef struct cf_forest cf_forest;
typedef struct cf_server cf_server;

/* One pixel sample: PixelInstance (src/curfil/random_tree_image.h:140-181) with the image
 * pointer replaced by an index into a dataset. 16 bytes. */
typedef struct cf_sample {
    uint16_t x, y;
    uint32_t image;
    float depth;      /* metres, Depth::getFloatValue() (image.h:146-149); <= 0 means invalid */
    uint8_t label;
    uint8_t flip;     /* HorizontalFlipSetting: 0 NoFlip, 1 Flip, 2 Both (random_tree.h:58-60) */
    uint16_t reserved;
} cf_sample;

/* SplitFunction result of evaluateBestSplits (random_tree_image.cpp:445-471). */
typedef struct cf_split {
    double score;
    int32_t feature;          /* index into the level's sorted candidate table */
    int32_t threshold_index;
    float threshold;
    int32_t flags;            /* bit 0: a candidate within 1e-13 of the best score was pushed out of a
                                 full four-entry candidate list, so the lowest-(threshold, feature)
                                 tie-break among near-ties is not guaranteed; 0 = exact. Which
                                 candidates meet in one list depends on the launch shape. */
} cf_split;

/* TrainingConfiguration (random_tree.h:187-493), the fields the hot path reads. */
typedef struct cf_train_config {
    int32_t random_seed;
    uint32_t samples_per_image;
    uint32_t feature_count;
    uint32_t min_sample_count;
    int32_t max_depth;
    uint16_t box_radius;        /* offset range ("boxRadius") */
    uint16_t region_size;       /* box half-size range ("regionSize") */
    uint16_t thresholds;
    uint16_t sampler;           /* cf_forest_train's classUniform sampler: 0 the reference's reservoir on the
                                   host (its RNG streams, one thread), 1 the device sampler of
                                   cf_sample_tree_pixels_device (project extension, deterministic) */
    int32_t num_threads;
    int32_t max_images;
    int32_t image_cache_size;
    uint32_t max_samples_per_batch;
    int32_t acceleration_mode;  /* 0 CPU_ONLY, 1 GPU_ONLY, 2 GPU_AND_CPU_COMPARE (random_tree.h:79-83) */
    int32_t use_cie_lab;
    int32_t use_depth_filling;
    int32_t use_depth_images;
    int32_t horizontal_flipping;
    int32_t subsampling_type;   /* 0 classUniform, 1 pixelUniform */
} cf_train_config;

/* ---------------------------------------------------------------------------------------------
 * Context and errors
 * ------------------------------------------------------------------------------------------- */
const char* cf_version(void);
/* Message of the last failed call on this thread; returns its full length. */
size_t cf_last_error(char* buffer, size_t length);
/* Replaces selectDevice/initDevice and the global streams (random_tree_image_gpu.cu:55-56,1722-1770). */
cf_status cf_context_create(int device, cf_context** out);
cf_status cf_context_destroy(cf_context* ctx);
/* Launch all work of this context on `stream` (a cudaStream_t); NULL restores the own stream. */
cf_status cf_context_set_stream(cf_context* ctx, void* stream);
cf_status cf_context_synchronize(cf_context* ctx);
/* Per-kernel CUDA-event timing (replaces utils::Profile, utils.h:159-203). */
cf_status cf_context_set_timing(cf_context* ctx, int enable);
cf_status cf_context_kernel_time(cf_context* ctx, const char* kernel, double* total_ms, int64_t* launches);
cf_status cf_context_reset_timing(cf_context* ctx);
/* Number of kernel launches issued by this context since creation. */
int64_t cf_context_launch_count(cf_context* ctx);
/* Name, SM count and compute capability of the context's device (e.g. to key tuning caches). */
cf_status cf_context_device(cf_context* ctx, char* name, size_t name_length, int* num_sms, int* cc_major,
                            int* cc_minor);

/* Launch shape of the level-batched split search used by every training call on this context.
 * Project extension with no reference counterpart (the reference's launch shapes are compile-time
 * constants, random_tree_image_gpu.cu:1455-1720). Read the current values with get, change fields,
 * write them back with set; set(NULL) restores the defaults. Results do not depend on the tuning,
 * only speed does. */
typedef struct cf_eval_tuning {
    int32_t features_per_tile;   /* features per shared-memory tile at most, 2..64 (default 16) */
    int32_t bins_budget_words;   /* histogram words per CTA, 1024..49152 (default 7168) */
    int32_t warp_aggregate;      /* 1: warp-aggregated shared increments, 0: plain atomics (default) */
    int32_t ctas_per_sm;         /* resident CTAs per SM the kernel is compiled for, 1..4 (default 3) */
    int32_t feature_granule;     /* work items cover a multiple of this many features, 1..64 (default 4) */
    float items_per_slot;        /* work items per resident CTA at most, (0, 8192] (default 2048) */
    int32_t sample_groups;       /* 0: each thread takes one sample through the tile's features; 1 (default):
                                    the lanes of a warp take (sample, feature) pairs of a few consecutive
                                    samples (neighbours in the image, so gathers share L1 lines) */
    int32_t min_item_evals;      /* feature evaluations per work item at least, 256..2^30 (default 16384): a
                                    level gets items_per_slot items per resident CTA or as many as hold this
                                    much work, whichever is fewer. Many items per node keep many CTAs on
                                    the same samples at once (their gathers share L2), but small items
                                    pay their setup more often */
    int32_t stage_bins;          /* 1 (default): when the integral images exceed the L2 cache, every level
                                    is searched in two passes: the threshold bins of every (sample,
                                    feature) are computed in frame order (the gathers of one frame's
                                    samples share L2) into a byte table, then histogrammed node by node
                                    (huge nodes in sample slices). 0: never; 2: always (T <= 255) */
    int32_t stage_max_mb;        /* device memory of the staged bin table at most, 1..65536 MiB (default 8192);
                                    a level whose table is larger runs in feature chunks */
    int32_t sample_order;        /* levels searched in one pass: 1 (default) reads a copy of the samples sorted
                                    by (node, frame, Morton code of the pixel) where the integral images
                                    exceed the L2 cache, so a CTA's samples lie in a compact patch and
                                    share L1 lines; 0: the level's order; 2: always sorted */
} cf_eval_tuning;
cf_status cf_context_get_tuning(cf_context* ctx, cf_eval_tuning* out);
cf_status cf_context_set_tuning(cf_context* ctx, const cf_eval_tuning* tuning);
/* Project-written autotuner (no reference counterpart): trains the given tree (as cf_train_tree,
 * level-batched) under candidate launch shapes, starting from the context's current one, by
 * coordinate descent over (sample_groups, warp_aggregate), bins_budget_words, items_per_slot,
 * feature_granule, min_item_evals, stage_bins, sample_order and features_per_tile,
 * timing the split search with the trainer's CUDA events (min over `repeats`). Every candidate must
 * yield the identical tree (else CF_ERR_STATE). The fastest shape is set on the context and returned
 * with its time; `start_ms` is the time of the starting shape, `trials` the shapes measured (either
 * may be NULL). On error the context keeps its previous shape. */
cf_status cf_autotune_split_search(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_classes,
                                   const cf_train_config* config, int tree_id, int32_t seed_counter, int repeats,
                                   cf_eval_tuning* best, double* best_ms, double* start_ms, int* trials);

/* ---------------------------------------------------------------------------------------------
 * Datasets: integral images resident in device memory
 * Replaces RGBDImage::calculateIntegral (image.cpp:531-556) and ImageCache (random_tree_image_gpu.cu:727-908).
 * ------------------------------------------------------------------------------------------- */
cf_status cf_dataset_create(cf_context* ctx, int num_images, int width, int height, cf_dataset** out);
cf_status cf_dataset_destroy(cf_dataset* ds);
/* Raw frames -> integral images on the GPU. rgb uint8 [count][H][W][3], depth_mm uint16 [count][H][W]
 * (0 = missing). `device_pointers` != 0 means both inputs already live in device memory. */
cf_status cf_dataset_upload_raw(cf_dataset* ds, int first, int count, const uint8_t* rgb,
                                const uint16_t* depth_mm, int device_pointers);
/* The same with the reference's image preprocessing: fill_depth = RGBDImage::fillDepth
 * (image.cpp:279-377, the caller's frames are not modified), cie_lab = colour in CIE L*a*b*
 * (image.cpp:89-96; the published CIE 1976 formulas with BT.709 primaries and D65 white, as the
 * reference's Vigra functor implements them for linear RGB). */
cf_status cf_dataset_upload_raw_ex(cf_dataset* ds, int first, int count, const uint8_t* rgb,
                                   const uint16_t* depth_mm, int device_pointers, int fill_depth, int cie_lab);
/* Frames smaller than the dataset's, as loadImages pads them to the largest frame
 * (LabeledRGBDImage::resizeImage, image.cpp:450-475, 796-800, 904-950): rgb uint8 [count][height][width][3]
 * and depth_mm [count][height][width] are preprocessed and integrated at their own size, then placed in
 * the top-left corner of the dataset's frames; the rest of each frame gets colour integral NaN and
 * depth integral {0, 0}, as RGBDImage::resizeImage leaves it. Labels are padded by the caller
 * (LabelImage::resizeImage, image.cpp:763-777, with the padding label of getPaddingLabel). */
cf_status cf_dataset_upload_raw_padded(cf_dataset* ds, int first, int count, int width, int height,
                                       const uint8_t* rgb, const uint16_t* depth_mm, int device_pointers,
                                       int fill_depth, int cie_lab);
/* RGBDImage::calculateIntegral (image.cpp:236-277, 531-556) of images in the reference's own layout:
 * colour float [count][3][H][W] (any float values, as setColor stores them) and depth int32
 * [count][2][H][W] (depth mm with 0 for invalid, valid 0/1, as setDepth stores them). Colour is summed
 * in double and rounded to float (identical to the reference's Kahan scan for integer-valued colours;
 * within the final float rounding otherwise), depth in 32-bit integers that wrap (box differences
 * stay exact). Outputs have the input layouts; host or device pointers. */
cf_status cf_integrate_planes(cf_context* ctx, int count, int width, int height, const float* color,
                              const int32_t* depth, float* color_integral, int32_t* depth_integral,
                              int device_pointers);
/* RGBDImage::fillDepth on depth frames uint16 [count][H][W], in place (host or device pointers). */
cf_status cf_fill_depth(cf_context* ctx, int count, int width, int height, uint16_t* depth_mm, int device_pointers);
/* The L*a*b* planes float [count][3][H][W] of RGB frames uint8 [count][H][W][3] (before integration). */
cf_status cf_rgb_to_cielab(cf_context* ctx, int count, int width, int height, const uint8_t* rgb, float* lab,
                           int device_pointers);
/* Already-integrated images in the reference layout: colour float [count][3][H][W], depth int32
 * [count][2][H][W] (sum in mm, valid count), e.g. from RGBDImage::getColorImage/getDepthImage. */
cf_status cf_dataset_upload_integral(cf_dataset* ds, int first, int count, const float* color,
                                     const int32_t* depth);
cf_status cf_dataset_download_integral(cf_dataset* ds, int first, int count, float* color, int32_t* depth);
cf_status cf_dataset_info(cf_dataset* ds, int* num_images, int* width, int* height);

/* ---------------------------------------------------------------------------------------------
 * ImageFeatureEvaluation (random_tree_image.h:988-1096), host buffers
 * Features are the int8 [11][F] table of ImageFeaturesAndThresholds (random_tree_image.h:635-912):
 * rows type, offset1X, offset1Y, offset2X, offset2Y, region1X, region1Y, region2X, region2Y,
 * channel1, channel2. Thresholds are float [T][F].
 * ------------------------------------------------------------------------------------------- */
/* featureResponseKernel (random_tree_image_gpu.cu:1455-1545): responses double [F][N]. */
cf_status cf_feature_responses(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_features,
                               const int8_t* features, double* responses);
/* calculateFeatureResponsesAndHistograms (random_tree_image_gpu.cu:1958-2135): counters uint32
 * [F][T][C][2] (0 = left, 1 = right), exact for any number of classes <= 256. */
cf_status cf_histograms(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_features,
                        int num_thresholds, const int8_t* features, const float* thresholds, int num_classes,
                        uint32_t* counters);
/* calculateScores (random_tree_image_gpu.cu:2137-2182): scores double [T][F] from counters
 * [F][T][C][2] and the node histogram [C]. */
cf_status cf_scores(cf_context* ctx, int num_classes, int num_features, int num_thresholds,
                    const uint32_t* counters, const uint32_t* node_histogram, double* scores);
/* Float lower/upper bounds [T][F] that enclose the scores cf_scores returns for the same counters
 * (left + right must equal the node histogram per class). Project extension with no reference
 * counterpart: the screening the level-batched split search applies before exact double scoring. */
cf_status cf_score_bounds(cf_context* ctx, int num_classes, int num_features, int num_thresholds,
                          const uint32_t* counters, const uint32_t* node_histogram, float* lower, float* upper);
/* generateRandomFeatures (random_tree_image_gpu.cu:1896-1956 + sortFeatures :1853-1894): the
 * candidate generator of the GPU path on a Philox4x32-10 stream, sorted by getSortKey. */
cf_status cf_generate_features(cf_dataset* ds, int num_samples, const cf_sample* samples, uint32_t seed,
                               int num_features, int num_thresholds, int box_radius, int region_size,
                               int use_depth_images, int8_t* features, float* thresholds);
/* evaluateBestSplits (random_tree_image.cpp:239-502) for all open nodes of one level in one
 * persistent launch. Node n owns samples [node_offsets[n], node_offsets[n+1]). The samples are
 * checked (image, pixel, label, flip) and the node histograms counted on up to 16 host threads while
 * the samples upload; an invalid sample fails the call with the index of the first one (as does
 * cf_generate_features, which checks its samples the same way). */
cf_status cf_evaluate_best_splits(cf_dataset* ds, int num_nodes, const int64_t* node_offsets,
                                  const cf_sample* samples, int num_classes, int num_features,
                                  int num_thresholds, const int8_t* features, const float* thresholds,
                                  cf_split* best);

/* cf_evaluate_best_splits that also returns the counts the level-batched kernel accumulated:
 * left_counts uint32 [M][F][T][C] (samples of node m, class c, with response <= threshold t), the
 * left half of the counters of calculateFeatureResponsesAndHistograms (random_tree_image_gpu.cu:1958-2135)
 * for every node of the level. For verification; training never materialises these counts. */
cf_status cf_level_left_counts(cf_dataset* ds, int num_nodes, const int64_t* node_offsets,
                               const cf_sample* samples, int num_classes, int num_features,
                               int num_thresholds, const int8_t* features, const float* thresholds,
                               cf_split* best, uint32_t* left_counts);
/* Allocation-free form of cf_evaluate_best_splits. No counterpart in the reference: it exists for
 * callers that cannot let a library allocate device memory (a host that owns all GPU memory through
 * its own pool, or a latency-critical loop where cudaMalloc/cudaFree would synchronise the device).
 * Every input and output is a DEVICE pointer the caller owns: integral images (colour float
 * [n][3][H][W], depth int32 pairs {sum, valid} [n][H][W]), samples, node histograms uint32 [M][C]
 * (flip-Both samples counted twice), the feature table int8 [11][F], thresholds float [T][F] and
 * best [M]; node_offsets [M+1] is a HOST array. Scratch lives in one fixed 16 MiB device array
 * compiled into the library, so this call allocates nothing; limits: M <= 65536 nodes, at most 65536
 * work items, F <= 16384, T <= 4096, F x T <= 2^20 (larger levels return CF_ERR_INVALID).
 * Preconditions, checked on the device before the split search runs (CF_ERR_INVALID, nothing
 * evaluated): every sample has image < num_images, x < width, y < height, flip <= 2 and a label
 * < num_classes that its node's histogram counts; no threshold is NaN. The histograms should equal
 * the nodes' class counts: other nonzero counts give meaningless scores but are not detected. The
 * first call on a device loads the module that holds the array (make it before any stream capture).
 * Calls share the array: calls that overlap on the GPU (other threads or streams) race and must be
 * serialised. */
cf_status cf_evaluate_best_splits_noalloc(cf_context* ctx, const float* color, const int32_t* depth,
                                          int num_images, int width, int height, int num_nodes,
                                          const int64_t* node_offsets, const cf_sample* samples,
                                          const uint32_t* node_histograms, int num_classes, int num_features,
                                          int num_thresholds, const int8_t* features, const float* thresholds,
                                          cf_split* best);

/* ---------------------------------------------------------------------------------------------
 * Tree training
 * ------------------------------------------------------------------------------------------- */
#define CF_TRAIN_LEVEL_BATCHED 0   /* all open nodes of a level in one persistent launch */
#define CF_TRAIN_PER_NODE 1        /* reference structure: per node responses -> histograms -> scores -> host argmax */

/* RandomTreeImage::train from a sample list (random_tree_image.cpp:746-824 after sampling) driving
 * RandomTreeTrain::train (random_tree.h:1249-1415). The level seeds are drawn from the tree's
 * RandomSource starting at *seed_counter, which is advanced as the reference advances it. */
cf_status cf_train_tree(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_classes,
                        const cf_train_config* config, int tree_id, int32_t* seed_counter, int mode,
                        cf_tree** out);
/* All-gather of `bytes` bytes from every process of a sharded training: recv receives world x bytes,
 * process r's contribution at offset r x bytes. Host buffers. Returns 0 on success. */
typedef int (*cf_allgather_fn)(const void* send, size_t bytes, void* recv, void* user);
/* One tree trained by `world` processes together (the reference trains a tree on one device; its
 * multi-device mode assigns whole trees, random_tree_image_gpu.cu:1727). Every process passes the
 * same dataset contents, samples, configuration, tree id and seed counter. Per level each process
 * evaluates its share of the level-batched work items (node x feature range; positions rank,
 * rank + world, ... of the largest-first order), and one call of `allgather` per level exchanges the
 * items' candidate lists. All processes then hold the same splits, route identically and return the
 * same tree, identical to cf_train_tree's (level-batched). The exchange is 88 bytes per work item
 * (about 2.5 MB per level at 200 frames x 2000 features). The tree's feature evaluation count is this
 * process's share. */
cf_status cf_train_tree_sharded(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_classes,
                                const cf_train_config* config, int tree_id, int32_t* seed_counter, int rank,
                                int world, cf_allgather_fn allgather, void* user, cf_tree** out);
/* One level of a tree's training on its own. The reference trains a level as one pass of the loop
 * body of RandomTreeTrain::train (random_tree.h:1262-1410): evaluateBestSplits for the level's open
 * nodes (random_tree_image.cpp:239-502), then routing of every sample into its child. There it has
 * no entry point of its own; here a level's input state (its node-contiguous samples, open nodes,
 * node histograms and level seed) is captured during a training and can be trained again, to
 * measure or compare the split search on a chosen level of a large tree without training the tree.
 * cf_train_tree_snapshots trains like cf_train_tree (level-batched) and returns a snapshot of each
 * listed level (root = 1) the tree reaches, in level order (*num_snapshots of them, at most
 * num_levels). Snapshots keep device memory (about 20 bytes per sample) and use their dataset's
 * training buffers: destroy them before the dataset. */
typedef struct cf_level_snapshot cf_level_snapshot;
cf_status cf_train_tree_snapshots(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_classes,
                                  const cf_train_config* config, int tree_id, int32_t* seed_counter, int num_levels,
                                  const int32_t* levels, cf_level_snapshot** snapshots, int* num_snapshots,
                                  cf_tree** out);
cf_status cf_level_snapshot_info(cf_level_snapshot* snapshot, int* level, int* num_nodes, int64_t* num_samples);
/* The level's node offsets [M + 1], samples [n] (host buffers, either may be NULL) and level seed:
 * the inputs of evaluateBestSplits for this level (cf_generate_features with that seed gives the
 * level's candidate table). */
cf_status cf_level_snapshot_export(cf_level_snapshot* snapshot, int64_t* node_offsets, cf_sample* samples,
                                   uint32_t* seed);
/* Trains the level again as the training loop does: candidate generation, the split search in `mode`
 * (CF_TRAIN_LEVEL_BATCHED or CF_TRAIN_PER_NODE) and routing into the next level's sample lists. best
 * (host [M], may be NULL) receives the splits; device_ms is the level's time on the device (CUDA
 * events), feature_evals = samples x features; next_nodes and next_samples describe the next level.
 * Any pointer may be NULL. The snapshot itself is not changed, so runs repeat exactly. */
cf_status cf_level_snapshot_run(cf_level_snapshot* snapshot, int mode, cf_split* best, double* device_ms,
                                int64_t* feature_evals, int* next_nodes, int64_t* next_samples);
cf_status cf_level_snapshot_destroy(cf_level_snapshot* snapshot);
/* RandomForestImage::train (random_forest_image.cpp:132-182) on raw host frames: GPU integral images,
 * class-uniform sampling (random_tree_image.cpp:911-1059, one host thread), block sort, then
 * cf_train_tree per tree. labels uint8 [n][H][W]; ignored[C] marks ignoredColors. */
cf_status cf_forest_train(cf_context* ctx, int num_images, int width, int height, const uint8_t* rgb,
                          const uint16_t* depth_mm, const uint8_t* labels, int num_classes,
                          const uint8_t* ignored, const cf_train_config* config, int num_trees, int mode,
                          cf_tree** trees);
/* The forest seed of RandomForestImage::train (random_forest_image.cpp:150-151): the first draw of
 * uniformSampler(0xFFFF) on RandomSource(random_seed). Tree t uses seed counter SEED + t. */
cf_status cf_forest_seed(int32_t random_seed, int32_t* seed);
/* Training pixels of one tree as RandomForestImage::train draws them (maxImages reservoir
 * random_forest_image.cpp:161-171, class prior random_tree_image.cpp:885-909, class- or
 * pixel-uniform sampling :840-1059 on one host thread, block sort :776-802). *seed_counter is the
 * tree's RandomSource counter and is advanced; prior[C] receives the class prior (may be NULL).
 * With out == NULL only *count is set. */
cf_status cf_sample_tree_pixels(int num_images, int width, int height, const uint8_t* labels,
                                const uint16_t* depth_mm, int num_classes, const uint8_t* ignored,
                                const cf_train_config* config, int num_trees, int32_t* seed_counter,
                                cf_sample* out, int64_t capacity, int64_t* count, uint32_t* prior);
/* The same on the device for classUniform (project extension; the reference's sampler is not
 * reproducible with several threads). Each eligible pixel (label not ignored, depth > 0) at
 * position k of the tree's image list and pixel p gets the key Philox4x32-10(key = (s, 0x53414D50),
 * counter = (k*H*W + p, 0, 0, 0)) word 0, s being the draw the reference's sampler takes from the
 * tree's RandomSource; every class keeps its per-class quota of pixels with the smallest
 * (key, k*H*W + p); samples are ordered by (image, label, y/10, x/10, y, x). Host inputs; the
 * seed counter advances as for cf_sample_tree_pixels. */
cf_status cf_sample_tree_pixels_device(cf_context* ctx, int num_images, int width, int height, const uint8_t* labels,
                                       const uint16_t* depth_mm, int num_classes, const uint8_t* ignored,
                                       const cf_train_config* config, int num_trees, int32_t* seed_counter,
                                       cf_sample* out, int64_t capacity, int64_t* count, uint32_t* prior);
/* RandomTree accessors (random_tree.h:499-1003). */
cf_status cf_tree_info(cf_tree* tree, int* num_nodes, int* num_classes, int* depth, int* tree_id);
/* Node arrays in breadth-first id order (index = nodeId - treeId); any pointer may be NULL.
 * level, left (-1 leaf; right child = left + 1), feature int8 [n][11], threshold, score, feature_id,
 * histogram uint32 [n][C], num_samples. */
cf_status cf_tree_export(cf_tree* tree, int32_t* level, int32_t* left, int8_t* feature, float* threshold,
                         double* score, int32_t* feature_id, uint32_t* histogram, uint32_t* num_samples);
cf_status cf_tree_import(int tree_id, int num_nodes, int num_classes, const int32_t* level, const int32_t* left,
                         const int8_t* feature, const float* threshold, const double* score,
                         const int32_t* feature_id, const uint32_t* histogram, cf_tree** out);
cf_status cf_tree_destroy(cf_tree* tree);
/* classLabelPriorDistribution of the tree (RandomTreeImage::getClassLabelPriorDistribution,
 * random_tree_image.h:1160-1163): pixel counts per class over its training images. */
cf_status cf_tree_prior(cf_tree* tree, uint32_t* prior, int capacity, int* count);
cf_status cf_tree_set_prior(cf_tree* tree, const uint32_t* prior, int count);
/* Per-level statistics of the last training of this tree: feature evaluations and device time. */
cf_status cf_tree_train_stats(cf_tree* tree, int64_t* feature_evals, double* device_ms, int* levels);
/* Per level of the last training: open nodes, their samples and the device time of the split search
 * (the reference logs per-level times, random_tree.h:1259,1411). Copies min(capacity, levels) entries. */
cf_status cf_tree_level_stats(cf_tree* tree, int capacity, int* num_levels, int32_t* nodes, int64_t* samples,
                              float* eval_ms);
/* Start of each level's split search in the last training, ms after the training's first device
 * work (CUDA events; for lining per-level times up with clock and power samples). */
cf_status cf_tree_level_starts(cf_tree* tree, int capacity, float* start_ms);

/* ---------------------------------------------------------------------------------------------
 * Prediction: RandomForestImage::normalizeHistograms + convertTree + predict
 * (random_forest_image.cpp:258-376; random_tree_image_gpu.cu:424-578, 1237-1453)
 * ------------------------------------------------------------------------------------------- */
/* Normalises every leaf histogram (detail::normalizeHistogram, random_tree.cpp:54-104) with the
 * class prior [C] (NULL: each tree's own prior) and packs the trees for the traversal kernel. */
cf_status cf_forest_create(cf_context* ctx, int num_trees, cf_tree* const* trees, const uint32_t* prior,
                           double histogram_bias, int use_labels_prior, cf_forest** out);
cf_status cf_forest_destroy(cf_forest* forest);
cf_status cf_forest_info(cf_forest* forest, int* num_trees, int* num_classes, int64_t* num_nodes);
/* Preprocessing of raw frames before prediction (cf_predict_host*, graphs, the server), as the
 * forest was trained: useDepthFilling and useCIELab of its TrainingConfiguration (default off). */
cf_status cf_forest_set_preprocessing(cf_forest* forest, int fill_depth, int cie_lab);
/* Dense prediction of `count` dataset images from `first`: probabilities float [count][C][H][W] and
 * labels uint8 [count][H][W], both DEVICE pointers (either may be NULL). */
cf_status cf_predict_dataset(cf_forest* forest, cf_dataset* ds, int first, int count, float* probabilities,
                             uint8_t* labels);
/* cf_predict_dataset with the results copied to HOST buffers (either may be NULL); the
 * RandomForestImage::predict form for images already integrated (random_forest_image.cpp:258-301). */
cf_status cf_predict_dataset_host(cf_forest* forest, cf_dataset* ds, int first, int count, float* probabilities,
                                  uint8_t* labels);
/* detail::normalizeHistogram (random_tree.cpp:54-104) of one histogram [C] with the class prior [C]:
 * h'_c = max(0, h_c - bias * sum h), divided by sum h', times prior_c / sum prior when
 * use_labels_prior. Host only (the reference normalises on the host once per tree). */
cf_status cf_normalize_histogram(int num_classes, const uint32_t* histogram, const uint32_t* prior,
                                 double histogram_bias, int use_labels_prior, double* out);
/* Same from raw host frames, results to host buffers (either may be NULL). */
cf_status cf_predict_host(cf_forest* forest, int count, int width, int height, const uint8_t* rgb,
                          const uint16_t* depth_mm, float* probabilities, uint8_t* labels);
/* The plain per-image launch form of classifyImage (random_tree_image_gpu.cu:1414-1453): per image,
 * one launch per tree accumulating into probabilities, then normalisation and argmax launches, each
 * followed by a stream synchronisation. Same results as cf_predict_dataset; kept as the baseline the
 * batched form is measured against. DEVICE pointers, either may be NULL. */
cf_status cf_predict_dataset_plain(cf_forest* forest, cf_dataset* ds, int first, int count, float* probabilities,
                                   uint8_t* labels);
/* The plain form from raw host frames as RandomForestImage::predict runs it on the GPU
 * (random_forest_image.cpp:258-301): per image, upload and integral images, the launches above,
 * then the full probabilities [C][H][W] and the labels copied back to the host (the probabilities
 * are copied even when `probabilities` is NULL, as there). HOST pointers. */
cf_status cf_predict_host_plain(cf_forest* forest, int count, int width, int height, const uint8_t* rgb,
                                const uint16_t* depth_mm, float* probabilities, uint8_t* labels);

/* A fixed batch of `count` raw frames (width x height) captured once as a CUDA graph: host-to-device
 * copy from pinned staging buffers, integral images, classification, results back to pinned buffers.
 * Project extension with no reference counterpart. Fill the buffers returned by
 * cf_predict_graph_buffers (rgb uint8 [count][H][W][3], depth uint16 [count][H][W]), call run, read
 * labels uint8 [count][H][W] and, when requested at creation, probabilities float [count][C][H][W].
 * Destroy the graph before its forest. */
typedef struct cf_predict_graph cf_predict_graph;
cf_status cf_predict_graph_create(cf_forest* forest, int count, int width, int height, int with_probabilities,
                                  cf_predict_graph** out);
cf_status cf_predict_graph_buffers(cf_predict_graph* graph, uint8_t** rgb, uint16_t** depth_mm, float** probabilities,
                                   uint8_t** labels);
cf_status cf_predict_graph_run(cf_predict_graph* graph);
cf_status cf_predict_graph_destroy(cf_predict_graph* graph);

/* ---------------------------------------------------------------------------------------------
 * Serving: continuous batching of mixed-resolution frames on a resident forest
 * (replaces the per-image test() loop, predict.cpp:209-375)
 * ------------------------------------------------------------------------------------------- */
typedef struct cf_server_config {
    int64_t hbm_budget_bytes;   /* admission limit for frames in flight */
    int32_t max_batch_frames;   /* frames per launch */
    int32_t max_pending;        /* queue length before submits are rejected */
    int32_t pipeline_depth;     /* batches in flight on the device */
    int32_t return_probabilities;
    int32_t policy;             /* admission order: 0 arrival; 1 smallest frame first, except that a request
                                   waiting longer than max_wait_ms goes first (no frame waits for ever) */
    float max_wait_ms;          /* age limit of policy 1 */
    int32_t device_priority;    /* 1: a batch holds frames of one size class (one class per factor 4 in pixels)
                                   and runs on a stream whose CUDA priority rises as the class's frames get
                                   smaller, so the thread blocks of small frames are scheduled ahead of those
                                   still waiting in a larger frame's launch; 0: one priority for all */
    float max_queue_ms;         /* load shedding: a request still queued this long after its submission is
                                   refused (cf_server_wait returns CF_ERR_REJECTED) instead of being served
                                   late; 0: no limit */
} cf_server_config;

typedef struct cf_request_stats {
    double submit_ms;      /* host clock at submit, ms since server start */
    double admitted_ms;
    double done_ms;
    int32_t batch_id;
    int32_t batch_frames;
} cf_request_stats;

cf_status cf_server_create(cf_forest* forest, const cf_server_config* config, cf_server** out);
cf_status cf_server_destroy(cf_server* server);
/* Copies the frame; returns at once with a request id. */
cf_status cf_server_submit(cf_server* server, int width, int height, const uint8_t* rgb, const uint16_t* depth_mm,
                           int64_t* request_id);
/* Waits (bounded) for a request; copies labels uint8 [H][W] and, if the server returns them,
 * probabilities float [C][H][W] (either pointer may be NULL). */
cf_status cf_server_wait(cf_server* server, int64_t request_id, double timeout_s, uint8_t* labels,
                         float* probabilities, cf_request_stats* stats);
cf_status cf_server_counters(cf_server* server, int64_t* submitted, int64_t* completed, int64_t* rejected,
                             int64_t* batches);

/* ---------------------------------------------------------------------------------------------
 * The learned part: a per-pixel refinement network on the forest's output (project extension; the
 * reference has no learned component, its nearest hook is the disabled leaf-histogram refinement,
 * random_forest_image.cpp:184-255). Input per pixel (D = 3C + 2): the forest's class probabilities,
 * their means over (2 radius1 + 1)^2 and (2 radius2 + 1)^2 boxes, depth in metres / 5 and a depth-valid
 * flag; one hidden ReLU layer; softmax cross-entropy; Adam. Parameters (float): W1 [hidden][D],
 * b1 [hidden], W2 [C][hidden], b2 [C].
 * ------------------------------------------------------------------------------------------- */
typedef struct cf_refiner cf_refiner;
typedef struct cf_refiner_config {
    int32_t hidden;             /* hidden units, 1..128 */
    int32_t radius1, radius2;   /* context box radii */
    int32_t epochs;
    int32_t batch;              /* pixels per Adam step */
    int32_t pixels_per_image;   /* training pixels drawn per frame, uniform over labelled pixels */
    float learning_rate;
    uint32_t seed;              /* initialisation, pixel draws and shuffling */
} cf_refiner_config;
cf_status cf_refiner_create(cf_context* ctx, int num_classes, const cf_refiner_config* config, cf_refiner** out);
cf_status cf_refiner_destroy(cf_refiner* refiner);
/* Trains on dataset frames [first, first + count) with host labels uint8 [count][H][W] (ignored[C]
 * marks classes left out, may be NULL); loss_per_epoch[epochs] receives the mean training loss. */
cf_status cf_refiner_train(cf_refiner* refiner, cf_forest* forest, cf_dataset* ds, int first, int count,
                           const uint8_t* labels, const uint8_t* ignored, float* loss_per_epoch);
/* Refined probabilities float [count][C][H][W] and labels uint8 [count][H][W], DEVICE pointers
 * (either may be NULL). */
cf_status cf_refiner_predict(cf_refiner* refiner, cf_forest* forest, cf_dataset* ds, int first, int count,
                             float* probabilities, uint8_t* labels);
/* Read (get) and/or replace (set, resets the optimiser) the num_params parameters; host pointers. */
cf_status cf_refiner_params(cf_refiner* refiner, float* get, const float* set, int* num_params);
/* Mean loss and its gradient over n given rows (features float [n][D], labels uint8 [n]), computed by
 * the training kernels; host pointers. */
cf_status cf_refiner_loss_grad(cf_refiner* refiner, int n, const float* features, const uint8_t* labels,
                               float* grad, double* loss);
/* The input rows of n pixels (xy int32 [n][2]) of one dataset frame; out float [n][D], host. */
cf_status cf_refiner_features(cf_refiner* refiner, cf_forest* forest, cf_dataset* ds, int frame, int n,
                              const int32_t* xy, float* out);

/* ---------------------------------------------------------------------------------------------
 * Tree files: gzip-compressed JSON (RandomTreeExport::writeJSON export.cpp:292-313,
 * RandomTreeImport::readJSON import.cpp:175-266)
 * ------------------------------------------------------------------------------------------- */
cf_status cf_tree_write_json(cf_tree* tree, const cf_train_config* config, const uint32_t* prior,
                             const char* path, int verbose);
cf_status cf_tree_read_json(const char* path, cf_train_config* config, uint32_t* prior, int prior_capacity,
                            cf_tree** out);

/* ---------------------------------------------------------------------------------------------
 * Evaluation (predict.cpp:45-207)
 * ------------------------------------------------------------------------------------------- */
/* calculatePixelAccuracy over `count` frames: prediction and ground truth uint8 [count][H][W], DEVICE
 * pointers when device_pointers != 0, else host pointers (copied in). Pixels whose true label is
 * marked in ignored[C] (may be NULL) are skipped unless include_void; accuracy = correct / (all
 * pixels if include_void, else counted pixels). confusion uint64 [C][C] [label][prediction] (host,
 * may be NULL) is incremented by the counted pixels. */
cf_status cf_pixel_accuracy(cf_context* ctx, int count, int width, int height, const uint8_t* prediction,
                            const uint8_t* ground_truth, int num_classes, const uint8_t* ignored, int include_void,
                            uint64_t* confusion, double* accuracy, int device_pointers);
/* ConfusionMatrix::normalize + averageClassAccuracy: rows normalised by their sums (empty rows stay
 * 0), the mean of the diagonal over the classes not ignored (all if include_void). normalized
 * double [C][C] may be NULL. Host only. */
cf_status cf_confusion_average_class_accuracy(int num_classes, const uint64_t* confusion, const uint8_t* ignored,
                                              int include_void, double* normalized, double* average);

/* ---------------------------------------------------------------------------------------------
 * Synthetic RGB-D frames (seeded Voronoi scenes) for tests and benchmarks
 * ------------------------------------------------------------------------------------------- */
cf_status cf_synthetic_frames(uint64_t seed, int num_images, int width, int height, int num_cells,
                              int num_classes, int void_class, uint8_t* rgb, uint16_t* depth_mm,
                              uint8_t* labels);
/* Frames first_index .. first_index + num_images - 1 of the same seeded sequence (frames are
 * independent given (seed, index); the class appearance depends on the seed only). */
cf_status cf_synthetic_frames_from(uint64_t seed, int first_index, int num_images, int width, int height,
                                   int num_cells, int num_classes, int void_class, uint8_t* rgb,
                                   uint16_t* depth_mm, uint8_t* labels);

#ifdef __cplusplus
}
#endif

#endif
