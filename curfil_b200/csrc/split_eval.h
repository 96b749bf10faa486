// Split search of one tree level: the level-batched persistent kernel and the reference-structured
// per-node kernels.
#pragma once

#include "features.h"

namespace cf {

// One open node of a level: its samples are [start, start + count) of the level's sample array.
struct NodeDesc {
    long long start;
    int count;
    int tree_index;
};

struct EvalItem {
    int node;
    int f_begin;
    int f_end;
    // chunks > 1: the item covers samples [s_begin, s_end) of the node and is one of `chunks` items of
    // group `group` (same node and features); each adds its counts to the group's histogram in global
    // memory, and the one that finishes last scores the merged counts
    int chunks;
    int s_begin;
    int s_end;
    int group;
    int chunk;   // position of this item's slice among its group's chunks (0 for whole-node items)
};

constexpr int kMaxCand = 4;

// Near-best candidates of one work item: every entry has best - score < 1e-13, sorted by
// (threshold, feature), at most kMaxCand lowest indices. `dropped` is the highest score of a
// candidate that was in the window when a full list pushed it out (-inf if none): the node's
// choice is exact unless a dropped score lies within the node's final window.
struct ItemCandidates {
    double best;
    double s[kMaxCand];
    int t[kMaxCand];
    int f[kMaxCand];
    int n;
    int pad;
    double dropped;
};

// Launch shape of level_eval (cf_eval_tuning of the context; 256 threads per CTA).
struct EvalTuning {
    int ft_max = 16;              // features per tile upper bound
    int bins_budget_words = 7168;   // shared-memory histogram budget per CTA (u32 words)
    int warp_aggregate = 1;       // __match_any_sync aggregation of the shared-memory increments
    int ctas_per_sm = 3;
    double items_per_slot = 2048.0; // work items per resident CTA at most
    int feature_granule = 4;      // a work item covers a multiple of this many features
    int sample_groups = 0;        // 1: lanes take (sample, feature) pairs of consecutive samples
    int min_item_evals = 16384;   // feature evaluations per work item at least
    int stage_bins = 1;           // 0 never, 1 when the integral images exceed L2, 2 always (levels without slices)
    int stage_max_mb = 8192;      // staged bin table size limit (MiB)
    int sample_order = 1;         // 0 level order, 1 Morton-sorted copy when the frames exceed L2, 2 always

    static EvalTuning of(cf_context* ctx);
};

// Work items of one level: node n is cut into feature ranges so that the level yields about
// items_per_slot items per resident CTA; order lists the items by decreasing work (samples x features).
// With chunk_features > 0 and fewer than kChunkItemsPerSlot items per resident CTA (the top levels,
// where one or a few nodes hold every sample), the items of nodes with at least 2 x kMinChunkSamples
// samples cover at most chunk_features features (one histogram tile) and are cut into sample chunks,
// for at most max_groups groups (nodes past the limit keep whole-node items); *n_groups receives the
// number of chunk groups. Chunked items come first in the order, chunk-major.
constexpr int kChunkItemsPerSlot = 4;
constexpr int kMinChunkSamples = 4096;
// Samples per chunk where a level is chunked: about eight frames' worth at 8000 samples per frame,
// whose integral images (6 MB per 640x480 frame) fit in L2 together. Chunked items are queued
// chunk-major (every group's first chunk, then every group's second, ...), so the resident CTAs all
// gather from the same few frames and the gathers hit L2 instead of DRAM.
constexpr int kChunkTargetSamples = 65536;
constexpr size_t kMaxChunkGroupBytes = size_t(512) << 20;   // merged histograms of one level's chunk groups
constexpr int kChunkBigNodeSamples = 4 * 65536;             // nodes this large are always cut into slices
void plan_level_items(const std::vector<int>& node_counts, int F, const EvalTuning& tuning, int slots,
                      std::vector<EvalItem>& items, std::vector<int>& range, std::vector<int>& order,
                      int chunk_features = 0, int* n_groups = nullptr, int max_groups = 0);

// Staged bins (deep levels): pass 1 computes the threshold bin of every (sample, feature) with the
// level's samples taken in frame and Morton order, so the resident CTAs gather from one or two frames
// at a time (L2 hits), and writes it to a byte table of 32-feature blocks, each [row][32 bytes];
// pass 2 is the split search reading its bins from the table. Rows are the level's samples node by
// node; the table holds at most stage_max_mb MiB, so a level whose table would be larger runs in
// feature chunks (multiples of kStageTile features), each pass 1 followed by the items of its features.
constexpr int kStageTile = 32;   // features per table block
// launch shape of the pass-2 search (level_eval reading staged bins)
constexpr int kStagedFeatures = 32;           // features per tile at most
constexpr int kStagedBinsWords = 12288;       // histogram words per CTA
constexpr double kStagedItemsPerSlot = 64.0;  // work items per resident CTA at most (16 and 256: the same)
// Splits every item at the chunk boundaries (multiples of `chunk` features) and orders the items
// chunk by chunk, largest first within a chunk; chunk_begin[c] is the first order position of chunk c.
void split_items_into_chunks(const std::vector<int>& node_counts, int chunk, int n_chunks,
                             std::vector<EvalItem>& items, std::vector<int>& range, std::vector<int>& order,
                             std::vector<int>& chunk_begin);

class LevelEvaluator {
public:
    // nodes_dev / node_hist_dev: M node descriptors and [M][C] histograms on the device;
    // node_counts: the M sample counts on the host (for work-item sizing).
    void evaluate(cf_context* ctx, const DsView& ds, const Sample* samples, const NodeDesc* nodes_dev,
                  const uint32_t* node_hist_dev, int M, const std::vector<int>& node_counts, int C,
                  const LevelFeatures& lf, cf_split* splits_dev, uint32_t* dump_left = nullptr);
    EvalTuning tuning;            // the context's tuning at the last evaluate call
    int64_t last_items = 0;
    int last_stage_chunks = 0;    // feature chunks of the staged bins at the last call (0: not staged)
    int64_t last_local_evals = 0; // feature evaluations this process ran at the last evaluate call

    // Sharding of a level's work items over `world` processes (each holding the same dataset,
    // samples and candidate table): this process evaluates the items at positions rank, rank+world,
    // ... of the work order, then one all-gather of the item candidate lists gives every process the
    // complete list, so the splits equal those of one process.
    struct Shard {
        int rank = 0, world = 1;
        cf_allgather_fn allgather = nullptr;
        void* user = nullptr;
    } shard;

private:
    void exchange(cf_context* ctx, int n_items);
    void stage_order(cf_context* ctx, const DsView& ds, const Sample* samples, const NodeDesc* nodes_dev, int M,
                     const std::vector<int>& node_counts, long long rows, bool by_node);
    std::vector<ItemCandidates> h_cands_, h_send_, h_recv_;
    std::vector<int> h_local_order_;
    DevArray<EvalItem> items_;
    DevArray<int> order_;
    DevArray<int> item_range_;   // [M + 1] first item of each node
    DevArray<ItemCandidates> cands_;
    DevArray<int> queue_;
    DevArray<uint32_t> group_bins_;   // [groups][bins budget] merged counts of chunked items
    DevArray<int> group_count_;       // [groups] chunks finished
    DevArray<unsigned char> node_consts_;   // [M] scoring constants of each node
    DevArray<uint8_t> stage_;         // [blocks of 32 features][rows][32] staged bins of one feature chunk
    DevArray<long long> row_base_;    // [M + 1] first row of each node
    DevArray<int> row_pos_;           // [rows] position of each row's sample in the level's array
    DevArray<uint8_t> row_label_;     // [rows] label of each row's sample
    DevArray<int> flip_both_;         // set when a sample of the level has flip 2
    DevArray<Sample> sorted_samples_; // [rows] the level's samples sorted by (node, frame, Morton code)
    DevArray<unsigned long long> pixel_key_, pixel_key_sorted_;   // (frame, Morton code of y, x) of each row
    DevArray<int> row_ids_, frame_order_;   // rows, and rows in pixel order
    DevArray<unsigned char> sort_temp_;
    std::vector<long long> h_row_base_;
    std::vector<int> h_chunk_begin_;
    std::vector<EvalItem> h_items_;
    std::vector<int> h_order_;
    std::vector<int> h_range_;
};

// Reference-structured evaluation of one node (featureResponseKernel -> aggregateHistogramsKernel
// -> scoreKernel -> host argmax), the "plain per-node" form.
class PlainNodeEvaluator {
public:
    void evaluate_node(cf_context* ctx, const DsView& ds, const Sample* samples_dev, long long start, int count,
                       const uint32_t* node_hist_dev, int C, const LevelFeatures& lf, int max_batch,
                       cf_split* split_dev_out, cf_split* split_host_out);
    // counters [F][T][C][2] for samples on the device (accumulated over batches)
    void histograms(cf_context* ctx, const DsView& ds, const Sample* samples_dev, long long start, int count, int C,
                    const int8_t* feat_table, const float* thr, int F, int T, int max_batch);
    DevArray<uint32_t> counters;
    DevArray<double> scores;
    DevArray<double> resp1, resp2;
    std::vector<double> h_scores;
};

void plain_responses(cf_context* ctx, const DsView& ds, const Sample* samples_dev, long long start, int count,
                     const int8_t* feat_table, int F, double* resp1, double* resp2);
// Float bounds [T][F] of the exact scores (the screening of level_eval), counters [F][T][C][2].
void score_bounds(cf_context* ctx, int C, int F, int T, const uint32_t* counters, const uint32_t* node_hist,
                  float* lower, float* upper);
void plain_scores(cf_context* ctx, int C, int F, int T, const uint32_t* counters, const uint32_t* node_hist,
                  double* scores);

// Host window argmax: highest score, ties (best - s < 1e-13) to the lowest (threshold, feature).
void host_window_argmax(const double* scores, int F, int T, int* best_f, int* best_t, double* best_s);

}  // namespace cf
