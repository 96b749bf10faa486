// Routing of a level's samples into the children of its nodes (random_tree.h:1296-1406) on the GPU.
#pragma once

#include "split_eval.h"

namespace cf {

// Trained-tree node arrays in device memory, breadth-first order (index = nodeId - treeId).
struct DevTree {
    int capacity = 0;
    int C = 0;
    DevArray<int32_t> level, left, feature_id;
    DevArray<int8_t> feature;     // [cap][11]
    DevArray<float> threshold;
    DevArray<double> score;
    DevArray<uint32_t> hist;      // [cap][C]
    DevArray<uint32_t> nsamp;
    void reserve(int cap, int C);
};

class Scanner {
public:
    // out[i] = sum(in[0..i)) for i in [0, n]; out[n] is the total.
    void exclusive(cf_context* ctx, const uint32_t* in, uint32_t* out, long long n);

private:
    void scan_level(cf_context* ctx, const uint32_t* in, uint32_t* out, long long n_in, long long n_out, size_t depth);
    // two buffers per recursion depth; a fixed array so references stay valid while recursing
    // (1024^8 elements is far beyond any sample count)
    static constexpr size_t kMaxDepth = 8;
    DevArray<uint32_t> temps_[2 * kMaxDepth];
};

struct RouteBuffers {
    DevArray<uint32_t> cntL, cntR, posL, posR;
    DevArray<uint8_t> code;
    DevArray<uint32_t> child_hist;    // [2M][C]
    DevArray<uint32_t> cont, cont_count, next_idx, next_off;
    DevArray<int> err;
    void reserve(long long n, int M, int C);
};

struct RouteResult {
    int next_nodes = 0;
    long long next_samples = 0;
    int empty_child = 0;
};

// Routes one level: writes the parents' splits and the 2M children into `tree` (children at
// tree indices next_tree_base + 2i, + 1), then, if `scatter`, gathers the samples of continuing
// children into samples_out / node_out and their descriptors into next_nodes / next_hist.
RouteResult route_level(cf_context* ctx, const DsView& ds, const Sample* samples, const int* sample_node, long long n,
                        const NodeDesc* nodes, int M, const cf_split* splits, const LevelFeatures& lf, int C,
                        int level, int min_samples, int next_tree_base, bool scatter, DevTree& tree,
                        RouteBuffers& rb, Scanner& scan, Sample* samples_out, int* node_out, NodeDesc* next_nodes,
                        uint32_t* next_hist);

}  // namespace cf
