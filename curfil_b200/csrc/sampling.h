// Device class-uniform sampling of training pixels (definition in sampling.cu).
#pragma once

#include <vector>

#include "host_rng.h"
#include "internal.h"

namespace cf {

// Raw label and depth frames resident on the device for sampling, with the sampler's own stream
// and scratch, so that sampling the next tree can overlap the training of the current one.
struct DeviceFrames {
    int n = 0, W = 0, H = 0;
    cudaStream_t stream = nullptr;
    DevArray<uint8_t> labels;    // [n][H][W]
    DevArray<uint16_t> depth;    // [n][H][W], millimetres, 0 = missing
    // scratch of sample_class_uniform_device
    DevArray<int> images;
    DevArray<uint8_t> ignored;
    DevArray<uint32_t> counts;
    DevArray<int> bad;
    DevArray<unsigned long long> cut, count;
    DevArray<uint4> candidates;
    // selection and ordering on the device (radix sorts)
    DevArray<uint32_t> idx_a, idx_b, class_count, class_start;
    DevArray<unsigned long long> key_a, key_b;
    DevArray<uint8_t> sort_temp;
    DevArray<cf_sample> out;

    DeviceFrames() = default;
    DeviceFrames(const DeviceFrames&) = delete;
    DeviceFrames& operator=(const DeviceFrames&) = delete;
    ~DeviceFrames() {
        if (stream) cudaStreamDestroy(stream);
    }
    void upload(cf_context* ctx, int num_images, int width, int height, const uint8_t* labels_host,
                const uint16_t* depth_host);
};

// classUniform samples of the listed images (image field = position in `images`), in the defined
// order; advances `rs` by the two draws the reference's sampler takes. prior (if given) receives the
// label histogram of the listed images. Runs on frames.stream; one call at a time per DeviceFrames.
std::vector<cf_sample> sample_class_uniform_device(cf_context* ctx, DeviceFrames& frames,
                                                   const std::vector<int>& images, const uint16_t* depth_host,
                                                   int C, const uint8_t* ignored, int subsample_count,
                                                   RandomSource& rs, uint8_t flip, std::vector<uint32_t>* prior);

// pixelUniform samples of the listed images in the reference's definition (its random streams: the
// image of each sample from one Sampler, its pixel from two fresh Samplers, redrawn while the label is
// ignored), drawn on the device, block-sorted as RandomTreeImage::train sorts them; image field =
// position in `images`. Advances `rs` as the reference does (1 + 2 x samples seeds).
std::vector<cf_sample> sample_pixel_uniform_device(cf_context* ctx, DeviceFrames& frames, const std::vector<int>& images,
                                                   int C, const uint8_t* ignored, int subsample_count, RandomSource& rs,
                                                   uint8_t flip, std::vector<uint32_t>* prior);

}  // namespace cf
