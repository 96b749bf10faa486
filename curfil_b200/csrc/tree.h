// Host-side trained tree (RandomTree, random_tree.h:499-1003) in breadth-first node arrays.
#pragma once

#include <vector>

#include "internal.h"

struct cf_tree {
    int tree_id = 0;
    int C = 0;
    int num_nodes = 0;
    std::vector<int32_t> level, left, feature_id;
    std::vector<int8_t> feature;      // [n][11]
    std::vector<float> threshold;
    std::vector<double> score;
    std::vector<uint32_t> hist;       // [n][C]
    std::vector<uint32_t> nsamp;
    std::vector<uint32_t> prior;      // classLabelPriorDistribution [C] (may be empty)
    // statistics of the training run
    int64_t feature_evals = 0;
    double device_ms = 0.0;
    int levels = 0;
    std::vector<int32_t> level_nodes;     // open nodes evaluated per level
    std::vector<int64_t> level_samples;   // samples of those nodes
    std::vector<float> level_eval_ms;     // device time of the split search per level
    std::vector<float> level_start_ms;    // start of each level's split search, ms after the tree's start

    void resize(int n) {
        num_nodes = n;
        level.resize(n);
        left.resize(n);
        feature_id.resize(n);
        feature.resize(static_cast<size_t>(n) * 11);
        threshold.resize(n);
        score.resize(n);
        hist.resize(static_cast<size_t>(n) * C);
        nsamp.resize(n);
    }
    int depth() const {
        int d = 0;
        for (int32_t l : level) d = l > d ? l : d;
        return d;
    }
};
