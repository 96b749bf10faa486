// Host-only check of the split search's work-item planner (plan_level_items): every (node, feature,
// sample) evaluation is covered exactly once, chunk groups are consistent (same node and features,
// contiguous sample slices in order, `chunks` members, at most one histogram tile of features), the
// group limit holds, and the work order is a permutation. Prints one line per case, "ok" or "FAIL".
#include <algorithm>
#include <cstdio>
#include <map>
#include <vector>

#include "../../curfil_b200/csrc/split_eval.h"

using namespace cf;

static int failures = 0;

static void check(const char* name, std::vector<int> counts, int F, int chunk_features, int slots, int max_groups,
                  int expect_groups) {
    EvalTuning t;
    t.ft_max = 32;
    t.bins_budget_words = 7168;
    t.items_per_slot = 64.0;
    t.feature_granule = 8;
    t.ctas_per_sm = 3;
    std::vector<EvalItem> items;
    std::vector<int> range, order;
    int groups = -1;
    plan_level_items(counts, F, t, slots, items, range, order, chunk_features, &groups, max_groups);
    long long evals = 0, expect = 0;
    for (int c : counts) expect += static_cast<long long>(c) * F;
    std::map<int, std::vector<EvalItem>> by_group;
    bool ok = true;
    for (size_t i = 0; i < items.size(); i++) {
        const EvalItem& it = items[i];
        evals += static_cast<long long>(it.s_end - it.s_begin) * (it.f_end - it.f_begin);
        if (it.chunks > 1) {
            by_group[it.group].push_back(it);
            if (it.f_end - it.f_begin > chunk_features) ok = false;
        } else if (it.group != -1 || it.s_begin != 0 || it.s_end != counts[it.node]) {
            ok = false;
        }
        if (static_cast<int>(i) < range[it.node] || static_cast<int>(i) >= range[it.node + 1]) ok = false;
    }
    for (auto& kv : by_group) {
        const std::vector<EvalItem>& v = kv.second;
        if (static_cast<int>(v.size()) != v[0].chunks) ok = false;
        for (size_t j = 0; j < v.size(); j++) {
            if (v[j].node != v[0].node || v[j].f_begin != v[0].f_begin || v[j].f_end != v[0].f_end) ok = false;
            if (v[j].s_begin != (j ? v[j - 1].s_end : 0)) ok = false;
        }
        if (v.back().s_end != counts[v[0].node]) ok = false;
    }
    if (static_cast<int>(by_group.size()) != groups || groups > max_groups) ok = false;
    if (expect_groups >= 0 && groups != expect_groups) ok = false;
    if (evals != expect) ok = false;
    std::vector<int> seen(items.size(), 0);
    for (int o : order) seen[o]++;
    for (int s : seen) ok = ok && s == 1;
    // chunked items first, chunk-major: (slice, group) never decreases along the order
    bool in_chunked = true;
    for (size_t q = 0; q < order.size(); q++) {
        const EvalItem& it = items[order[q]];
        if (it.chunks > 1) {
            if (!in_chunked) ok = false;
            if (q > 0) {
                const EvalItem& pv = items[order[q - 1]];
                if (pv.chunks > 1 && (pv.chunk > it.chunk || (pv.chunk == it.chunk && pv.group > it.group))) ok = false;
            }
            if (it.s_end - it.s_begin > std::max(kChunkTargetSamples, counts[it.node] / 2)) ok = false;
        } else {
            in_chunked = false;
        }
    }
    if (!ok) failures++;
    std::printf("%s: items %zu groups %d %s\n", name, items.size(), groups, ok ? "ok" : "FAIL");
}

int main() {
    const int slots = 148 * 3, big = 1 << 20;
    // bench workload: 266 600 samples, 2000 features x 20 thresholds, 40 classes (8-feature tiles)
    check("root", {266600}, 2000, 8, slots, big, 250);
    check("level 2", {133000, 133600}, 2000, 8, slots, big, 500);
    check("level 3", {70000, 63000, 66000, 67600}, 2000, 8, slots, big, 1000);
    check("level 4 (enough items)", std::vector<int>(8, 33325), 2000, 8, slots, big, 0);
    check("no chunking requested", {266600}, 2000, 0, slots, big, 0);
    check("8 M samples, 4000 features, 5-feature tiles", {8000000}, 4000, 5, slots, big, 800);
    check("small nodes stay whole", {5000, 9000, 100, 0}, 2000, 8, slots, big, 250);
    check("fewer features than a granule", {200000}, 7, 8, slots, big, 1);
    check("one feature", {200000}, 1, 1, slots, big, 1);
    // group limit: 64 MB of 7168-word histograms, and of 20 200-word ones (200 classes x 101 bins)
    check("root under the 64 MB limit", {266600}, 2000, 8, slots, (64 << 20) / (4 * 7168), 250);
    check("over the limit: whole nodes", {266600, 200000}, 4000, 1, slots, (64 << 20) / (4 * 20200), 0);
    check("limit 0", {266600}, 2000, 8, slots, 0, 0);
    std::printf("%d failures\n", failures);
    return failures == 0 ? 0 : 1;
}
