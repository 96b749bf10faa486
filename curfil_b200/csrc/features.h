// Candidate-feature tables of one tree level in device memory.
#pragma once

#include "device_math.cuh"
#include "internal.h"

namespace cf {

struct LevelFeatures {
    int F = 0, T = 0;
    DevArray<int8_t> raw_feat;     // [11][F] unsorted
    DevArray<float> raw_thr;       // [T][F] unsorted
    DevArray<int32_t> keys;        // [F]
    DevArray<int8_t> feat;         // [11][F] sorted (ImageFeaturesAndThresholds layout)
    DevArray<float> thr;           // [T][F] sorted
    DevArray<FeatParams> packs;    // [F]
    DevArray<float> sorted_thr;    // [F][T] thresholds of each feature in ascending order
    DevArray<uint16_t> ranks;      // [F][T] position of threshold t in that order
    void reserve(int F, int T);
};

// Generates, sorts and prepares the level's candidates from `num_samples` device samples.
void generate_level_features(cf_context* ctx, const DsView& ds, const Sample* samples, uint32_t num_samples,
                             uint32_t seed, int box_radius, int region_size, int use_depth, LevelFeatures& lf);

// Builds packs / sorted_thr / ranks from lf.feat and lf.thr (for injected tables).
void prepare_eval_features(cf_context* ctx, LevelFeatures& lf);

DsView view_of(const cf_dataset* ds);

// Preprocessing of raw frames (useDepthFilling, useCIELab of TrainingConfiguration).
constexpr int kPreFillDepth = 1;
constexpr int kPreCieLab = 2;

// Integral images of `count` raw frames (device pointers). With kPreFillDepth the depth frames are
// filled IN PLACE first (RGBDImage::fillDepth), so `depth_dev` must then be a buffer the caller owns;
// with kPreCieLab the colour integral is that of the L*a*b* image.
void integrate_frames(cf_context* ctx, const uint8_t* rgb_dev, uint16_t* depth_dev, int count, int W, int H,
                      float* color_out, int2* depth_out, cudaStream_t stream = nullptr, int preprocess = 0);

// preprocess.cu
void fill_depth_frames(cf_context* ctx, uint16_t* depth, int count, int W, int H, cudaStream_t stream);
void rgb_to_lab(cf_context* ctx, const uint8_t* rgb, int count, int W, int H, float* lab, cudaStream_t stream);
void lab_color_integral(cf_context* ctx, const uint8_t* rgb, int count, int W, int H, float* color_out,
                        cudaStream_t stream);

}  // namespace cf
