// Forest resident on the device for dense prediction.
#pragma once

#include <map>
#include <tuple>

#include "device_math.cuh"
#include "internal.h"
#include "tree.h"

namespace cf {

// 16-byte packed node: split parameters, threshold, and a meta word
//   leaf:  bit 31 set, bits 0-30 = row of the leaf histogram table
//   split: bits 0-25 = left child (tree-local index, right = left + 1), bit 26 = feature type,
//          bits 27-28 = channel1, bits 29-30 = channel2
struct __align__(16) PackedNode {
    int8_t o1x, o1y, o2x, o2y;
    int8_t r1x, r1y, r2x, r2y;
    float threshold;
    uint32_t meta;
};

// One frame of a prediction launch.
struct FrameDesc {
    const float* color;    // [3][H][W] integral
    const int2* depth;     // [H][W] integral {sum, valid}
    float* probs;          // [C][H][W] or null
    uint8_t* labels;       // [H][W] or null
    int width, height;
    int first_block;       // first CTA of this frame in the launch
    int pad;
};

void classify_frames(cf_context* ctx, const cf_forest* forest, const FrameDesc* frames_dev, int num_frames,
                     int total_blocks, cudaStream_t stream = nullptr);
int classify_blocks_for(int width, int height);

}  // namespace cf

struct cf_forest {
    cf_context* ctx = nullptr;
    int num_trees = 0;
    int C = 0;
    int64_t num_nodes = 0;
    int cache_per_tree = 0;          // top nodes of each tree staged in shared memory
    int preprocess = 0;              // kPreFillDepth | kPreCieLab applied to raw frames before prediction
    std::vector<int> tree_base;      // first node of each tree in `nodes`
    cf::DevArray<cf::PackedNode> nodes;
    cf::DevArray<int> d_tree_base;
    cf::DevArray<float> leaves;      // [L][C] normalised histograms (float, as convertTree stores them)
    int64_t num_leaves = 0;
    // scratch of cf_predict_host
    cf::DevArray<uint8_t> raw_rgb;
    cf::DevArray<uint16_t> raw_depth;
    cf::DevArray<float> color;
    cf::DevArray<int2> depth;
    cf::DevArray<float> probs;
    cf::DevArray<uint8_t> labels;
    cf::DevArray<cf::FrameDesc> frames;
    std::vector<cf::FrameDesc> h_frames;
};
