// Autotuner of the split search's launch shape (cf_eval_tuning).
//
// The reference fixes its launch shapes at compile time (random_tree_image_gpu.cu:1455-1720). Here the
// shape that is fastest depends on the workload (classes x thresholds decide how many features fit a
// shared-memory tile, node sizes decide how finely a level must be cut into work items) and on the
// L1/shared-memory split of the GPU. The tuner trains the caller's tree under candidate shapes, takes
// the device time of the split search (the per-level CUDA events of the trainer), and keeps the
// fastest by coordinate descent over the sample mapping and increment aggregation, the histogram
// budget, the work items per CTA slot, the feature granule and the tile width. Every candidate must
// produce the identical tree; a difference is an error, never a silent choice.
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "internal.h"
#include "tree.h"

namespace {

bool same_tree(const cf_tree* a, const cf_tree* b) {
    if (a->num_nodes != b->num_nodes || a->left != b->left || a->feature != b->feature || a->hist != b->hist ||
        a->feature_id != b->feature_id)
        return false;
    for (int i = 0; i < a->num_nodes; i++)
        if (a->left[i] >= 0 && std::memcmp(&a->threshold[i], &b->threshold[i], sizeof(float)) != 0) return false;
    return true;
}

void check(cf_status s) {
    if (s == CF_OK) return;
    char buf[1024];
    cf_last_error(buf, sizeof(buf));
    cf::fail(s, std::string("autotune: ") + buf);
}

struct TreeDeleter {
    void operator()(cf_tree* t) const { cf_tree_destroy(t); }
};

}  // namespace

extern "C" cf_status cf_autotune_split_search(cf_dataset* ds, int num_samples, const cf_sample* samples,
                                              int num_classes, const cf_train_config* config, int tree_id,
                                              int32_t seed_counter, int repeats, cf_eval_tuning* best,
                                              double* best_ms, double* start_ms, int* trials) {
    cf_context* ctx = nullptr;
    cf_eval_tuning original{};
    const cf_status st = cf::guard([&] {
        CF_REQUIRE(ds && samples && config && best, "cf_autotune_split_search: NULL argument");
        CF_REQUIRE(repeats >= 1 && repeats <= 16, "cf_autotune_split_search: repeats must be in [1, 16]");
        check(cf_context_get_tuning(ds->ctx, &original));
        ctx = ds->ctx;
        std::unique_ptr<cf_tree, TreeDeleter> reference;
        int count = 0;
        // device time of the split search of one training (min over repeats)
        auto measure = [&](const cf_eval_tuning& t) {
            check(cf_context_set_tuning(ctx, &t));
            double ms = std::numeric_limits<double>::infinity();
            for (int r = 0; r < repeats; r++) {
                int32_t counter = seed_counter;
                cf_tree* raw = nullptr;
                check(cf_train_tree(ds, num_samples, samples, num_classes, config, tree_id, &counter,
                                    CF_TRAIN_LEVEL_BATCHED, &raw));
                std::unique_ptr<cf_tree, TreeDeleter> tree(raw);
                double sum = 0;
                for (float x : tree->level_eval_ms) sum += x;
                ms = std::min(ms, sum);
                if (!reference) reference = std::move(tree);
                else if (!same_tree(reference.get(), tree.get()))
                    cf::fail(CF_ERR_STATE, "autotune: a launch shape changed the trained tree");
            }
            count++;
            return ms;
        };
        cf_eval_tuning cur = original;
        {   // warm-up: the first training allocates the trainer's buffers
            int32_t counter = seed_counter;
            cf_tree* raw = nullptr;
            check(cf_train_tree(ds, num_samples, samples, num_classes, config, tree_id, &counter,
                                CF_TRAIN_LEVEL_BATCHED, &raw));
            cf_tree_destroy(raw);
        }
        double cur_ms = measure(cur);
        if (start_ms) *start_ms = cur_ms;
        const int budgets[] = {4096, 6144, 7168, 8192, 10240, 12288};
        const float slots[] = {64.0f, 256.0f, 1024.0f, 2048.0f, 4096.0f};
        const int granules[] = {4, 8, 16};
        const int min_evals[] = {4096, 16384, 65536};
        const int tiles[] = {16, 32};
        for (int pass = 0; pass < 2; pass++) {
            bool improved = false;
            auto consider = [&](const cf_eval_tuning& cand) {
                if (std::memcmp(&cand, &cur, sizeof(cand)) == 0) return;
                const double ms = measure(cand);
                if (ms < cur_ms * 0.99) {   // keep a shape only for a clear gain
                    cur = cand;
                    cur_ms = ms;
                    improved = true;
                }
            };
            for (int g = 0; g < 2; g++)
                for (int agg = 0; agg < 2; agg++) {
                    cf_eval_tuning c = cur;
                    c.sample_groups = g;
                    c.warp_aggregate = agg;
                    consider(c);
                }
            for (int v : budgets) {
                cf_eval_tuning c = cur;
                c.bins_budget_words = v;
                consider(c);
            }
            for (float v : slots) {
                cf_eval_tuning c = cur;
                c.items_per_slot = v;
                consider(c);
            }
            for (int v : granules) {
                cf_eval_tuning c = cur;
                c.feature_granule = v;
                consider(c);
            }
            for (int v : min_evals) {
                cf_eval_tuning c = cur;
                c.min_item_evals = v;
                consider(c);
            }
            for (int v = 0; v <= 1; v++) {
                cf_eval_tuning c = cur;
                c.stage_bins = v;
                consider(c);
                c = cur;
                c.sample_order = v;
                consider(c);
            }
            for (int v : tiles) {
                cf_eval_tuning c = cur;
                c.features_per_tile = v;
                consider(c);
            }
            if (!improved) break;
        }
        check(cf_context_set_tuning(ctx, &cur));
        *best = cur;
        if (best_ms) *best_ms = cur_ms;
        if (trials) *trials = count;
    });
    if (st != CF_OK && ctx) cf_context_set_tuning(ctx, &original);
    return st;
}
