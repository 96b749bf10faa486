// Breadth-first tree training on the GPU (RandomTreeTrain::train, random_tree.h:1249-1415, with
// ImageFeatureEvaluation::evaluateBestSplits, random_tree_image.cpp:239-502) and the
// ImageFeatureEvaluation entry points of the C-ABI.
//
// Per level, all on the device: candidate generation from the level's samples, the split search
// (level-batched persistent launch, or node by node in the reference's structure), and routing
// into the next level's node-contiguous sample array. The host only draws the level seed, sizes
// the work items from the node counts and checks the empty-child flag.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <thread>

#include "host_rng.h"
#include "route.h"
#include "tree.h"

namespace cf {

namespace {

void validate_config(const cf_train_config* cfg) {
    CF_REQUIRE(cfg != nullptr, "training configuration is NULL");
    CF_REQUIRE(cfg->feature_count >= 1, "featureCount must be >= 1");
    CF_REQUIRE(cfg->thresholds >= 1, "thresholds must be >= 1");
    CF_REQUIRE(cfg->max_depth >= 1, "maxDepth must be >= 1");
    CF_REQUIRE(cfg->box_radius > 0, "boxRadius must be > 0");
    CF_REQUIRE(cfg->region_size > 0, "regionSize must be > 0");
    CF_REQUIRE(cfg->max_images <= 0 || cfg->max_images >= cfg->image_cache_size,
               "illegal configuration: maxImages must not be lower than imageCacheSize");
}

void check_sample(const cf_dataset* ds, const cf_sample& x, long long i, int C) {
    CF_REQUIRE(x.image < static_cast<uint32_t>(ds->n), "sample " + std::to_string(i) + ": image index out of range");
    CF_REQUIRE(x.x < ds->width && x.y < ds->height, "sample " + std::to_string(i) + ": pixel outside the image");
    CF_REQUIRE(x.label < C, "sample " + std::to_string(i) + ": label >= number of classes");
    CF_REQUIRE(x.flip <= 2, "sample " + std::to_string(i) + ": unknown flip setting");
}

void validate_samples(const cf_dataset* ds, const cf_sample* s, long long n, int C) {
    for (long long i = 0; i < n; i++) check_sample(ds, s[i], i, C);
}

// validate_samples over host threads (the host-buffer entry points take millions of samples per
// call), and with `hist` the class histogram [M][C] of the nodes whose samples are
// [offsets[m], offsets[m + 1]) (a flip-2 sample counts twice). Each thread takes a contiguous range of
// samples: nodes inside its range are its own rows of `hist`, the (at most two) nodes its range shares
// with its neighbours are counted in private rows and added afterwards. On invalid input the error is
// that of the first invalid sample, as validate_samples reports it.
void scan_samples(const cf_dataset* ds, const cf_sample* s, long long n, int C, const int64_t* offsets, int M,
                  uint32_t* hist) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int T = static_cast<int>(std::max<long long>(1, std::min<long long>(std::min<unsigned>(hw, 16u), n >> 18)));
    if (T == 1 && !hist) {
        validate_samples(ds, s, n, C);
        return;
    }
    struct Part {
        long long a = 0, b = 0, bad = -1;
        int first = 0, last = 0;
        std::vector<uint32_t> head, tail;
    };
    std::vector<Part> parts(T);
    const uint32_t nimg = static_cast<uint32_t>(ds->n);
    auto work = [&](Part& p) {
        int node = 0;
        if (hist) {
            node = static_cast<int>(std::upper_bound(offsets, offsets + M + 1, static_cast<int64_t>(p.a)) - offsets) - 1;
            p.first = node;
            p.last = static_cast<int>(std::upper_bound(offsets, offsets + M + 1, static_cast<int64_t>(p.b - 1)) - offsets) - 1;
            p.head.assign(C, 0);
            if (p.last != p.first) p.tail.assign(C, 0);
        }
        for (long long i = p.a; i < p.b; i++) {
            const cf_sample& x = s[i];
            if (!(x.image < nimg && x.x < ds->width && x.y < ds->height && x.label < C && x.flip <= 2)) {
                p.bad = i;
                return;
            }
            if (!hist) continue;
            while (offsets[node + 1] <= i) node++;
            const uint32_t add = x.flip == 2 ? 2u : 1u;
            if (node == p.first) p.head[x.label] += add;
            else if (node == p.last) p.tail[x.label] += add;
            else hist[static_cast<size_t>(node) * C + x.label] += add;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < T; t++) {
        parts[t].a = n * t / T;
        parts[t].b = n * (t + 1) / T;
        if (t + 1 < T) pool.emplace_back(work, std::ref(parts[t]));
    }
    work(parts[T - 1]);
    for (std::thread& th : pool) th.join();
    for (const Part& p : parts)   // in sample order: the first invalid sample's error
        if (p.bad >= 0) check_sample(ds, s[p.bad], p.bad, C);
    if (!hist) return;
    for (const Part& p : parts) {
        if (p.a >= p.b) continue;
        for (int c = 0; c < C; c++) hist[static_cast<size_t>(p.first) * C + c] += p.head[c];
        if (p.last != p.first)
            for (int c = 0; c < C; c++) hist[static_cast<size_t>(p.last) * C + c] += p.tail[c];
    }
}

void validate_thresholds(const float* thr, long long n) {
    for (long long i = 0; i < n; i++) CF_REQUIRE(!std::isnan(thr[i]), "thresholds must not be NaN");
}

}  // namespace

}  // namespace cf

// The input state of one level of a tree's training (the loop body of RandomTreeTrain::train,
// random_tree.h:1262-1410): the level's node-contiguous samples, their node indices, the open nodes
// and their histograms, and the level seed, so the level can be trained again on its own.
struct cf_level_snapshot {
    cf_dataset* ds = nullptr;
    int level = 0, M = 0, C = 0, tree_next = 0;
    long long n = 0;
    uint32_t seed = 0;
    cf_train_config cfg{};
    std::vector<int> counts;              // samples per open node (host)
    std::vector<int64_t> offsets;         // [M + 1] node offsets into the level's samples (host)
    cf::DevArray<cf::Sample> samples;
    cf::DevArray<int> snode;
    cf::DevArray<cf::NodeDesc> nodes;
    cf::DevArray<uint32_t> hist;
    // results of the last run
    float last_ms = 0;
    int64_t last_evals = 0;
    int next_nodes = 0;
    long long next_samples = 0;
};

namespace cf {

class TreeTrainer {
public:
    TreeTrainer(cf_dataset* ds, int C, const cf_train_config& cfg, int mode) : ds_(ds), C_(C), cfg_(cfg), mode_(mode) {}
    void rebind(cf_dataset* ds) { ds_ = ds; }   // the buffers are the dataset-independent state
    void configure(int C, const cf_train_config& cfg, int mode) {
        C_ = C;
        cfg_ = cfg;
        mode_ = mode;
    }

    cf_tree* train(const cf_sample* host_samples, int N, int tree_id, int32_t* seed_counter) {
        cf_context* ctx = ds_->ctx;
        make_current(ctx);
        CF_REQUIRE(N > 0, "training needs at least one sample");
        CF_REQUIRE(C_ >= 1 && C_ <= 256, "number of classes must be in [1, 256]");
        validate_samples(ds_, host_samples, N, C_);
        const int F = static_cast<int>(cfg_.feature_count), T = cfg_.thresholds;
        bool any_both = false;
        std::vector<uint32_t> root_hist(C_, 0);
        for (int i = 0; i < N; i++) {
            root_hist[host_samples[i].label] += host_samples[i].flip == 2 ? 2 : 1;
            any_both |= host_samples[i].flip == 2;
        }
        const long long cap = static_cast<long long>(N) * (any_both ? 2 : 1);
        CF_REQUIRE(2 * cap + 1 < (1LL << 31), "too many samples for one tree");
        samples_[0].reserve(cap);
        samples_[1].reserve(cap);
        snode_[0].reserve(cap);
        snode_[1].reserve(cap);
        nodes_[0].reserve(cap);
        nodes_[1].reserve(cap);
        hist_[0].reserve(static_cast<size_t>(cap) * C_);
        hist_[1].reserve(static_cast<size_t>(cap) * C_);
        splits_.reserve(cap);
        tree_.reserve(static_cast<int>(2 * cap + 1), C_);
        lf_.reserve(F, T);

        cudaStream_t st = ctx->stream;
        CF_CUDA_CHECK(cudaMemcpyAsync(samples_[0].get(), host_samples, sizeof(cf_sample) * N, cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemsetAsync(snode_[0].get(), 0, sizeof(int) * N, st));
        NodeDesc root{0, N, 0};
        CF_CUDA_CHECK(cudaMemcpyAsync(nodes_[0].get(), &root, sizeof(NodeDesc), cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(hist_[0].get(), root_hist.data(), sizeof(uint32_t) * C_, cudaMemcpyHostToDevice, st));
        // root record
        {
            const int32_t lvl = 1, lft = -1, fid = -1;
            const float nanf = std::nanf("");
            const double nand = std::nan("");
            const uint32_t ns = N;
            int8_t zeros[11] = {0};
            CF_CUDA_CHECK(cudaMemcpyAsync(tree_.level.get(), &lvl, 4, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(tree_.left.get(), &lft, 4, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(tree_.feature_id.get(), &fid, 4, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(tree_.threshold.get(), &nanf, 4, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(tree_.score.get(), &nand, 8, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(tree_.nsamp.get(), &ns, 4, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(tree_.feature.get(), zeros, 11, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(tree_.hist.get(), root_hist.data(), sizeof(uint32_t) * C_, cudaMemcpyHostToDevice, st));
        }
        cudaEvent_t ev0, ev1;
        CF_CUDA_CHECK(cudaEventCreate(&ev0));
        CF_CUDA_CHECK(cudaEventCreate(&ev1));
        CF_CUDA_CHECK(cudaEventRecord(ev0, st));

        const DsView ds = view_of(ds_);
        RandomSource rs(seed_counter);
        int cur = 0;
        int M = 1;
        long long n = N;
        int level = 1;
        int tree_next = 1;
        int64_t evals = 0;
        int levels = 0;
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> level_events;
        std::vector<int32_t> level_nodes;
        std::vector<int64_t> level_samples;
        std::vector<NodeDesc> h_nodes;
        std::vector<int> counts;
        while (M > 0 && level < cfg_.max_depth) {
            // evaluateBestSplits: one seed per level from the tree's random source
            const uint32_t seed = static_cast<uint32_t>(rs.uniform(0xFFFFFF).next());
            generate_level_features(ctx, ds, samples_[cur].get(), static_cast<uint32_t>(n), seed, cfg_.box_radius,
                                    cfg_.region_size, cfg_.use_depth_images, lf_);
            h_nodes.resize(M);
            CF_CUDA_CHECK(cudaMemcpyAsync(h_nodes.data(), nodes_[cur].get(), sizeof(NodeDesc) * M,
                                          cudaMemcpyDeviceToHost, st));
            CF_CUDA_CHECK(cudaStreamSynchronize(st));
            counts.resize(M);
            for (int i = 0; i < M; i++) counts[i] = h_nodes[i].count;
            if (captured_ && std::find(capture_.begin(), capture_.end(), level) != capture_.end())
                captured_->push_back(snapshot(cur, level, M, n, seed, tree_next, counts, h_nodes));
            cudaEvent_t le0, le1;
            CF_CUDA_CHECK(cudaEventCreate(&le0));
            CF_CUDA_CHECK(cudaEventCreate(&le1));
            CF_CUDA_CHECK(cudaEventRecord(le0, st));
            level_events.emplace_back(le0, le1);
            level_nodes.push_back(M);
            level_samples.push_back(n);
            if (mode_ == CF_TRAIN_PER_NODE) {
                for (int i = 0; i < M; i++)
                    plain_.evaluate_node(ctx, ds, samples_[cur].get(), h_nodes[i].start, h_nodes[i].count,
                                         hist_[cur].get() + static_cast<size_t>(i) * C_, C_, lf_,
                                         static_cast<int>(cfg_.max_samples_per_batch), splits_.get() + i, nullptr);
            } else {
                eval_.evaluate(ctx, ds, samples_[cur].get(), nodes_[cur].get(), hist_[cur].get(), M, counts, C_, lf_,
                               splits_.get());
            }
            CF_CUDA_CHECK(cudaEventRecord(le1, st));
            evals += eval_.shard.world > 1 ? eval_.last_local_evals : n * F;
            levels++;
            const bool scatter = level + 1 < cfg_.max_depth;
            const int nxt = 1 - cur;
            RouteResult rr = route_level(ctx, ds, samples_[cur].get(), snode_[cur].get(), n, nodes_[cur].get(), M,
                                         splits_.get(), lf_, C_, level, static_cast<int>(cfg_.min_sample_count),
                                         tree_next, scatter, tree_, rb_, scan_, samples_[nxt].get(), snode_[nxt].get(),
                                         nodes_[nxt].get(), hist_[nxt].get());
            if (rr.empty_child) {
                cudaEventDestroy(ev0);
                cudaEventDestroy(ev1);
                fail(CF_ERR_EMPTY_CHILD, "no samples in left or right node (tree " + std::to_string(tree_id) +
                                             ", level " + std::to_string(level) + ")");
            }
            tree_next += 2 * M;
            if (!scatter) break;
            cur = nxt;
            M = rr.next_nodes;
            n = rr.next_samples;
            level++;
        }
        CF_CUDA_CHECK(cudaEventRecord(ev1, st));
        CF_CUDA_CHECK(cudaEventSynchronize(ev1));
        float ms = 0;
        CF_CUDA_CHECK(cudaEventElapsedTime(&ms, ev0, ev1));
        cudaEventDestroy(ev1);

        auto* t = new cf_tree();
        t->tree_id = tree_id;
        t->C = C_;
        t->resize(tree_next);
        const int nn = tree_next;
        CF_CUDA_CHECK(cudaMemcpyAsync(t->level.data(), tree_.level.get(), 4 * nn, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(t->left.data(), tree_.left.get(), 4 * nn, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(t->feature_id.data(), tree_.feature_id.get(), 4 * nn, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(t->feature.data(), tree_.feature.get(), 11 * static_cast<size_t>(nn),
                                      cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(t->threshold.data(), tree_.threshold.get(), 4 * nn, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(t->score.data(), tree_.score.get(), 8 * nn, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(t->hist.data(), tree_.hist.get(), sizeof(uint32_t) * C_ * static_cast<size_t>(nn),
                                      cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(t->nsamp.data(), tree_.nsamp.get(), 4 * nn, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        t->feature_evals = evals;
        t->device_ms = ms;
        t->levels = levels;
        t->level_nodes = level_nodes;
        t->level_samples = level_samples;
        for (auto& pr : level_events) {
            float lms = 0;
            cudaEventElapsedTime(&lms, pr.first, pr.second);
            t->level_eval_ms.push_back(lms);
            float start = 0;
            cudaEventElapsedTime(&start, ev0, pr.first);
            t->level_start_ms.push_back(start);
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
        cudaEventDestroy(ev0);
        return t;
    }

    // Levels (root = 1) whose input state the next train() call copies into snapshots.
    void capture(const std::vector<int>& levels, std::vector<cf_level_snapshot*>* out) {
        capture_ = levels;
        captured_ = out;
    }

    // One level trained again from its snapshot, as the training loop runs it: candidate
    // generation with the level seed, the split search (level-batched or per node) and routing of
    // the samples into the next level's node-contiguous lists (into this trainer's buffers, which the
    // snapshot never reads). best (host, [M]) receives the splits when not NULL.
    void run_level(cf_level_snapshot* s, int mode, cf_split* best) {
        cf_context* ctx = ds_->ctx;
        make_current(ctx);
        configure(s->C, s->cfg, mode);
        const int F = static_cast<int>(cfg_.feature_count), T = cfg_.thresholds, M = s->M;
        const long long n = s->n;
        samples_[1].reserve(n);
        snode_[1].reserve(n);
        nodes_[1].reserve(2 * static_cast<size_t>(M));
        hist_[1].reserve(2 * static_cast<size_t>(M) * C_);
        splits_.reserve(M);
        if (tree_.capacity < s->tree_next + 2 * M) tree_.reserve(s->tree_next + 2 * M, C_);
        lf_.reserve(F, T);
        cudaStream_t st = ctx->stream;
        cudaEvent_t e0, e1;
        CF_CUDA_CHECK(cudaEventCreate(&e0));
        CF_CUDA_CHECK(cudaEventCreate(&e1));
        struct Events {
            cudaEvent_t a, b;
            ~Events() {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
        } evs{e0, e1};
        const DsView ds = view_of(ds_);
        CF_CUDA_CHECK(cudaEventRecord(e0, st));
        generate_level_features(ctx, ds, s->samples.get(), static_cast<uint32_t>(n), s->seed, cfg_.box_radius,
                                cfg_.region_size, cfg_.use_depth_images, lf_);
        if (mode == CF_TRAIN_PER_NODE) {
            for (int i = 0; i < M; i++)
                plain_.evaluate_node(ctx, ds, s->samples.get(), s->offsets[i], s->counts[i],
                                     s->hist.get() + static_cast<size_t>(i) * C_, C_, lf_,
                                     static_cast<int>(cfg_.max_samples_per_batch), splits_.get() + i, nullptr);
        } else {
            eval_.evaluate(ctx, ds, s->samples.get(), s->nodes.get(), s->hist.get(), M, s->counts, C_, lf_,
                           splits_.get());
        }
        const bool scatter = s->level + 1 < cfg_.max_depth;
        RouteResult rr = route_level(ctx, ds, s->samples.get(), s->snode.get(), n, s->nodes.get(), M, splits_.get(), lf_,
                                     C_, s->level, static_cast<int>(cfg_.min_sample_count), s->tree_next, scatter,
                                     tree_, rb_, scan_, samples_[1].get(), snode_[1].get(), nodes_[1].get(),
                                     hist_[1].get());
        CF_CUDA_CHECK(cudaEventRecord(e1, st));
        CF_CUDA_CHECK(cudaEventSynchronize(e1));
        if (rr.empty_child)
            fail(CF_ERR_EMPTY_CHILD, "no samples in left or right node (level " + std::to_string(s->level) + ")");
        CF_CUDA_CHECK(cudaEventElapsedTime(&s->last_ms, e0, e1));
        s->last_evals = n * F;
        s->next_nodes = rr.next_nodes;
        s->next_samples = rr.next_samples;
        if (best)
            CF_CUDA_CHECK(cudaMemcpy(best, splits_.get(), sizeof(cf_split) * M, cudaMemcpyDeviceToHost));
    }

    LevelEvaluator eval_;
    // device buffers of the host-buffer entry points (evaluateBestSplits, candidate generation), kept
    // so that repeated calls on a dataset do not allocate and free their inputs each time
    struct HostCall {
        DevArray<Sample> samples;
        DevArray<NodeDesc> nodes;
        DevArray<uint32_t> hist;
        DevArray<cf_split> best;
        LevelFeatures lf;
    } host_;

private:
    cf_level_snapshot* snapshot(int cur, int level, int M, long long n, uint32_t seed, int tree_next,
                                const std::vector<int>& counts, const std::vector<NodeDesc>& h_nodes) {
        std::unique_ptr<cf_level_snapshot> s(new cf_level_snapshot());
        s->ds = ds_;
        s->level = level;
        s->M = M;
        s->C = C_;
        s->n = n;
        s->seed = seed;
        s->tree_next = tree_next;
        s->cfg = cfg_;
        s->counts = counts;
        s->offsets.resize(M + 1);
        for (int i = 0; i < M; i++) s->offsets[i] = h_nodes[i].start;
        s->offsets[M] = n;
        s->samples.reserve(n);
        s->snode.reserve(n);
        s->nodes.reserve(M);
        s->hist.reserve(static_cast<size_t>(M) * C_);
        cudaStream_t st = ds_->ctx->stream;
        CF_CUDA_CHECK(cudaMemcpyAsync(s->samples.get(), samples_[cur].get(), sizeof(Sample) * n, cudaMemcpyDeviceToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(s->snode.get(), snode_[cur].get(), sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(s->nodes.get(), nodes_[cur].get(), sizeof(NodeDesc) * M, cudaMemcpyDeviceToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(s->hist.get(), hist_[cur].get(), sizeof(uint32_t) * M * C_, cudaMemcpyDeviceToDevice,
                                      st));
        return s.release();
    }

    std::vector<int> capture_;
    std::vector<cf_level_snapshot*>* captured_ = nullptr;
    cf_dataset* ds_;
    int C_;
    cf_train_config cfg_;
    int mode_;
    DevArray<cf_sample> samples_raw_;
    DevArray<Sample> samples_[2];
    DevArray<int> snode_[2];
    DevArray<NodeDesc> nodes_[2];
    DevArray<uint32_t> hist_[2];
    DevArray<cf_split> splits_;
    DevTree tree_;
    LevelFeatures lf_;
    RouteBuffers rb_;
    Scanner scan_;
    PlainNodeEvaluator plain_;
};

// The dataset's trainer (created on first use) holds the device buffers, allocated once, not per tree.
TreeTrainer* acquire_trainer(cf_dataset* ds, int C, const cf_train_config& cfg, int mode) {
    if (ds->trainer == nullptr) {
        // the buffers of a destroyed dataset's trainer, if the context keeps some
        cf_context* ctx = ds->ctx;
        std::lock_guard<std::mutex> lock(ctx->mu);
        if (ctx->spare_trainer) {
            ds->trainer = ctx->spare_trainer;
            ds->trainer_free = ctx->spare_trainer_free;
            ctx->spare_trainer = nullptr;
            ctx->spare_trainer_free = nullptr;
            static_cast<TreeTrainer*>(ds->trainer)->rebind(ds);
        }
    }
    if (ds->trainer == nullptr) {
        ds->trainer = new TreeTrainer(ds, C, cfg, mode);
        ds->trainer_free = [](void* p) { delete static_cast<TreeTrainer*>(p); };
    }
    return static_cast<TreeTrainer*>(ds->trainer);
}

cf_tree* train_tree(cf_dataset* ds, const cf_sample* samples, int N, int C, const cf_train_config& cfg, int tree_id,
                    int32_t* seed_counter, int mode, const LevelEvaluator::Shard* shard) {
    TreeTrainer* trainer = acquire_trainer(ds, C, cfg, mode);
    trainer->configure(C, cfg, mode);
    struct Reset {
        TreeTrainer* t;
        ~Reset() { t->eval_.shard = LevelEvaluator::Shard(); }
    } reset{trainer};
    trainer->eval_.shard = shard ? *shard : LevelEvaluator::Shard();
    return trainer->train(samples, N, tree_id, seed_counter);
}

}  // namespace cf

// ================================================================================================
// C-ABI
// ================================================================================================
using namespace cf;

namespace {

struct Uploaded {
    DevArray<Sample> samples;
    DevArray<int8_t> feat;
    DevArray<float> thr;
};

void upload_samples(cf_context* ctx, DevArray<Sample>& dst, const cf_sample* src, long long n) {
    dst.reserve(std::max<long long>(n, 1));
    if (n > 0)
        CF_CUDA_CHECK(cudaMemcpyAsync(dst.get(), src, sizeof(cf_sample) * n, cudaMemcpyHostToDevice, ctx->stream));
}

}  // namespace

extern "C" {

cf_status cf_feature_responses(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_features,
                               const int8_t* features, double* responses) {
    return guard([&] {
        CF_REQUIRE(ds && samples && features && responses, "cf_feature_responses: NULL argument");
        CF_REQUIRE(num_samples > 0 && num_features > 0, "cf_feature_responses: empty input");
        cf_context* ctx = ds->ctx;
        make_current(ctx);
        validate_samples(ds, samples, num_samples, 256);
        Uploaded u;
        upload_samples(ctx, u.samples, samples, num_samples);
        u.feat.reserve(static_cast<size_t>(11) * num_features);
        CF_CUDA_CHECK(cudaMemcpyAsync(u.feat.get(), features, 11 * static_cast<size_t>(num_features),
                                      cudaMemcpyHostToDevice, ctx->stream));
        DevArray<double> r1, r2;
        r1.reserve(static_cast<size_t>(num_features) * num_samples);
        r2.reserve(static_cast<size_t>(num_features) * num_samples);
        plain_responses(ctx, view_of(ds), u.samples.get(), 0, num_samples, u.feat.get(), num_features, r1.get(), r2.get());
        CF_CUDA_CHECK(cudaMemcpyAsync(responses, r1.get(), sizeof(double) * num_features * num_samples,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_histograms(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_features, int num_thresholds,
                        const int8_t* features, const float* thresholds, int num_classes, uint32_t* counters) {
    return guard([&] {
        CF_REQUIRE(ds && samples && features && thresholds && counters, "cf_histograms: NULL argument");
        CF_REQUIRE(num_samples > 0 && num_features > 0 && num_thresholds > 0, "cf_histograms: empty input");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_histograms: classes must be in [1, 256]");
        cf_context* ctx = ds->ctx;
        make_current(ctx);
        validate_samples(ds, samples, num_samples, num_classes);
        validate_thresholds(thresholds, static_cast<long long>(num_features) * num_thresholds);
        Uploaded u;
        upload_samples(ctx, u.samples, samples, num_samples);
        u.feat.reserve(static_cast<size_t>(11) * num_features);
        u.thr.reserve(static_cast<size_t>(num_thresholds) * num_features);
        CF_CUDA_CHECK(cudaMemcpyAsync(u.feat.get(), features, 11 * static_cast<size_t>(num_features),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(u.thr.get(), thresholds, sizeof(float) * num_features * num_thresholds,
                                      cudaMemcpyHostToDevice, ctx->stream));
        PlainNodeEvaluator pe;
        pe.histograms(ctx, view_of(ds), u.samples.get(), 0, num_samples, num_classes, u.feat.get(), u.thr.get(),
                      num_features, num_thresholds, 50000);
        CF_CUDA_CHECK(cudaMemcpyAsync(counters, pe.counters.get(),
                                      sizeof(uint32_t) * num_features * num_thresholds * num_classes * 2,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_scores(cf_context* ctx, int num_classes, int num_features, int num_thresholds, const uint32_t* counters,
                    const uint32_t* node_histogram, double* scores) {
    return guard([&] {
        CF_REQUIRE(ctx && counters && node_histogram && scores, "cf_scores: NULL argument");
        CF_REQUIRE(num_classes >= 1 && num_features > 0 && num_thresholds > 0, "cf_scores: empty input");
        make_current(ctx);
        const size_t nc = static_cast<size_t>(num_features) * num_thresholds * num_classes * 2;
        DevArray<uint32_t> c, h;
        DevArray<double> s;
        c.reserve(nc);
        h.reserve(num_classes);
        s.reserve(static_cast<size_t>(num_features) * num_thresholds);
        CF_CUDA_CHECK(cudaMemcpyAsync(c.get(), counters, sizeof(uint32_t) * nc, cudaMemcpyHostToDevice, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(h.get(), node_histogram, sizeof(uint32_t) * num_classes, cudaMemcpyHostToDevice,
                                      ctx->stream));
        plain_scores(ctx, num_classes, num_features, num_thresholds, c.get(), h.get(), s.get());
        CF_CUDA_CHECK(cudaMemcpyAsync(scores, s.get(), sizeof(double) * num_features * num_thresholds,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_score_bounds(cf_context* ctx, int num_classes, int num_features, int num_thresholds,
                          const uint32_t* counters, const uint32_t* node_histogram, float* lower, float* upper) {
    return guard([&] {
        CF_REQUIRE(ctx && counters && node_histogram && lower && upper, "cf_score_bounds: NULL argument");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256 && num_features > 0 && num_thresholds > 0,
                   "cf_score_bounds: empty input or more than 256 classes");
        make_current(ctx);
        const size_t nc = static_cast<size_t>(num_features) * num_thresholds * num_classes * 2;
        const size_t ns = static_cast<size_t>(num_features) * num_thresholds;
        for (size_t i = 0; i < nc; i += 2) {
            const size_t c = (i / 2) % num_classes;
            CF_REQUIRE(static_cast<uint64_t>(counters[i]) + counters[i + 1] == node_histogram[c],
                       "cf_score_bounds: left + right counts must equal the node histogram");
        }
        DevArray<uint32_t> c, h;
        DevArray<float> lo, up;
        c.reserve(nc);
        h.reserve(num_classes);
        lo.reserve(ns);
        up.reserve(ns);
        CF_CUDA_CHECK(cudaMemcpyAsync(c.get(), counters, sizeof(uint32_t) * nc, cudaMemcpyHostToDevice, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(h.get(), node_histogram, sizeof(uint32_t) * num_classes, cudaMemcpyHostToDevice,
                                      ctx->stream));
        score_bounds(ctx, num_classes, num_features, num_thresholds, c.get(), h.get(), lo.get(), up.get());
        CF_CUDA_CHECK(cudaMemcpyAsync(lower, lo.get(), sizeof(float) * ns, cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(upper, up.get(), sizeof(float) * ns, cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_generate_features(cf_dataset* ds, int num_samples, const cf_sample* samples, uint32_t seed,
                               int num_features, int num_thresholds, int box_radius, int region_size,
                               int use_depth_images, int8_t* features, float* thresholds) {
    return guard([&] {
        CF_REQUIRE(ds && samples && features && thresholds, "cf_generate_features: NULL argument");
        CF_REQUIRE(num_samples > 0 && num_features > 0 && num_thresholds > 0, "cf_generate_features: empty input");
        cf_context* ctx = ds->ctx;
        make_current(ctx);
        TreeTrainer* tr = acquire_trainer(ds, 1, cf_train_config{}, CF_TRAIN_LEVEL_BATCHED);
        TreeTrainer::HostCall& hc = tr->host_;
        upload_samples(ctx, hc.samples, samples, num_samples);   // overlaps the check below
        scan_samples(ds, samples, num_samples, 256, nullptr, 0, nullptr);
        LevelFeatures& lf = hc.lf;
        lf.reserve(num_features, num_thresholds);
        generate_level_features(ctx, view_of(ds), hc.samples.get(), static_cast<uint32_t>(num_samples), seed, box_radius,
                                region_size, use_depth_images, lf);
        CF_CUDA_CHECK(cudaMemcpyAsync(features, lf.feat.get(), 11 * static_cast<size_t>(num_features),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(thresholds, lf.thr.get(), sizeof(float) * num_features * num_thresholds,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

}  // extern "C"

namespace {

// evaluateBestSplits on host buffers; with `left_counts` the kernel also reports its left counts
// [M][F][T][C] (class = label).
void evaluate_level_host(cf_dataset* ds, int num_nodes, const int64_t* node_offsets, const cf_sample* samples,
                         int num_classes, int num_features, int num_thresholds, const int8_t* features,
                         const float* thresholds, cf_split* best, uint32_t* left_counts) {
    {
        CF_REQUIRE(ds && node_offsets && samples && features && thresholds && best, "cf_evaluate_best_splits: NULL argument");
        CF_REQUIRE(num_nodes > 0 && num_features > 0 && num_thresholds > 0, "cf_evaluate_best_splits: empty input");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_evaluate_best_splits: classes must be in [1, 256]");
        cf_context* ctx = ds->ctx;
        make_current(ctx);
        const long long n = node_offsets[num_nodes];
        CF_REQUIRE(node_offsets[0] == 0 && n > 0, "cf_evaluate_best_splits: node offsets must start at 0");
        std::vector<NodeDesc> nodes(num_nodes);
        std::vector<int> counts(num_nodes);
        for (int i = 0; i < num_nodes; i++) {
            CF_REQUIRE(node_offsets[i + 1] > node_offsets[i], "cf_evaluate_best_splits: every node needs samples");
            CF_REQUIRE(node_offsets[i + 1] - node_offsets[i] < (1LL << 31), "cf_evaluate_best_splits: node too large");
            nodes[i] = NodeDesc{node_offsets[i], static_cast<int>(node_offsets[i + 1] - node_offsets[i]), i};
            counts[i] = nodes[i].count;
        }
        TreeTrainer* tr = acquire_trainer(ds, num_classes, cf_train_config{}, CF_TRAIN_LEVEL_BATCHED);
        TreeTrainer::HostCall& hc = tr->host_;
        // the copy runs while the host checks the samples and counts the node histograms; nothing reads
        // the copy before they pass
        upload_samples(ctx, hc.samples, samples, n);
        std::vector<uint32_t> hist(static_cast<size_t>(num_nodes) * num_classes, 0);
        scan_samples(ds, samples, n, num_classes, node_offsets, num_nodes, hist.data());
        validate_thresholds(thresholds, static_cast<long long>(num_features) * num_thresholds);
        DevArray<NodeDesc>& d_nodes = hc.nodes;
        DevArray<uint32_t>& d_hist = hc.hist;
        DevArray<cf_split>& d_best = hc.best;
        d_nodes.reserve(num_nodes);
        d_hist.reserve(hist.size());
        d_best.reserve(num_nodes);
        CF_CUDA_CHECK(cudaMemcpyAsync(d_nodes.get(), nodes.data(), sizeof(NodeDesc) * num_nodes, cudaMemcpyHostToDevice,
                                      ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(d_hist.get(), hist.data(), sizeof(uint32_t) * hist.size(), cudaMemcpyHostToDevice,
                                      ctx->stream));
        LevelFeatures& lf = hc.lf;
        lf.reserve(num_features, num_thresholds);
        CF_CUDA_CHECK(cudaMemcpyAsync(lf.feat.get(), features, 11 * static_cast<size_t>(num_features),
                                      cudaMemcpyHostToDevice, ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(lf.thr.get(), thresholds, sizeof(float) * num_features * num_thresholds,
                                      cudaMemcpyHostToDevice, ctx->stream));
        prepare_eval_features(ctx, lf);
        LevelEvaluator& ev = tr->eval_;
        DevArray<uint32_t> d_left;
        const size_t n_left = static_cast<size_t>(num_nodes) * num_features * num_thresholds * num_classes;
        if (left_counts) {
            d_left.reserve(n_left);
            CF_CUDA_CHECK(cudaMemsetAsync(d_left.get(), 0, sizeof(uint32_t) * n_left, ctx->stream));
        }
        ev.evaluate(ctx, view_of(ds), hc.samples.get(), d_nodes.get(), d_hist.get(), num_nodes, counts, num_classes,
                    lf, d_best.get(), left_counts ? d_left.get() : nullptr);
        CF_CUDA_CHECK(cudaMemcpyAsync(best, d_best.get(), sizeof(cf_split) * num_nodes, cudaMemcpyDeviceToHost,
                                      ctx->stream));
        if (left_counts)
            CF_CUDA_CHECK(cudaMemcpyAsync(left_counts, d_left.get(), sizeof(uint32_t) * n_left, cudaMemcpyDeviceToHost,
                                          ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    }
}

}  // namespace

extern "C" {

cf_status cf_evaluate_best_splits(cf_dataset* ds, int num_nodes, const int64_t* node_offsets, const cf_sample* samples,
                                  int num_classes, int num_features, int num_thresholds, const int8_t* features,
                                  const float* thresholds, cf_split* best) {
    return guard([&] {
        evaluate_level_host(ds, num_nodes, node_offsets, samples, num_classes, num_features, num_thresholds, features,
                            thresholds, best, nullptr);
    });
}

cf_status cf_level_left_counts(cf_dataset* ds, int num_nodes, const int64_t* node_offsets, const cf_sample* samples,
                               int num_classes, int num_features, int num_thresholds, const int8_t* features,
                               const float* thresholds, cf_split* best, uint32_t* left_counts) {
    return guard([&] {
        CF_REQUIRE(left_counts, "cf_level_left_counts: left_counts is NULL");
        evaluate_level_host(ds, num_nodes, node_offsets, samples, num_classes, num_features, num_thresholds, features,
                            thresholds, best, left_counts);
    });
}

cf_status cf_train_tree(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_classes,
                        const cf_train_config* config, int tree_id, int32_t* seed_counter, int mode, cf_tree** out) {
    return guard([&] {
        CF_REQUIRE(ds && samples && seed_counter && out, "cf_train_tree: NULL argument");
        validate_config(config);
        CF_REQUIRE(mode == CF_TRAIN_LEVEL_BATCHED || mode == CF_TRAIN_PER_NODE, "cf_train_tree: unknown mode");
        *out = train_tree(ds, samples, num_samples, num_classes, *config, tree_id, seed_counter, mode, nullptr);
    });
}

cf_status cf_train_tree_sharded(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_classes,
                                const cf_train_config* config, int tree_id, int32_t* seed_counter, int rank,
                                int world, cf_allgather_fn allgather, void* user, cf_tree** out) {
    return guard([&] {
        CF_REQUIRE(ds && samples && seed_counter && out, "cf_train_tree_sharded: NULL argument");
        validate_config(config);
        CF_REQUIRE(world >= 1 && rank >= 0 && rank < world, "cf_train_tree_sharded: rank must be in [0, world)");
        CF_REQUIRE(world == 1 || allgather != nullptr, "cf_train_tree_sharded: no all-gather function");
        LevelEvaluator::Shard shard;
        shard.rank = rank;
        shard.world = world;
        shard.allgather = allgather;
        shard.user = user;
        *out = train_tree(ds, samples, num_samples, num_classes, *config, tree_id, seed_counter,
                          CF_TRAIN_LEVEL_BATCHED, &shard);
    });
}

cf_status cf_train_tree_snapshots(cf_dataset* ds, int num_samples, const cf_sample* samples, int num_classes,
                                  const cf_train_config* config, int tree_id, int32_t* seed_counter, int num_levels,
                                  const int32_t* levels, cf_level_snapshot** snapshots, int* num_snapshots,
                                  cf_tree** out) {
    return guard([&] {
        CF_REQUIRE(ds && samples && seed_counter && out && num_snapshots, "cf_train_tree_snapshots: NULL argument");
        CF_REQUIRE(num_levels >= 0 && (num_levels == 0 || (levels && snapshots)),
                   "cf_train_tree_snapshots: levels and snapshots are needed for num_levels > 0");
        validate_config(config);
        std::vector<int> want(levels, levels + num_levels);
        for (int l : want) CF_REQUIRE(l >= 1, "cf_train_tree_snapshots: levels start at 1 (the root)");
        std::vector<cf_level_snapshot*> got;
        TreeTrainer* trainer = acquire_trainer(ds, num_classes, *config, CF_TRAIN_LEVEL_BATCHED);
        struct Disarm {
            TreeTrainer* t;
            std::vector<cf_level_snapshot*>* got;
            bool ok = false;
            ~Disarm() {
                t->capture({}, nullptr);
                if (!ok)
                    for (auto* p : *got) delete p;
            }
        } disarm{trainer, &got};
        trainer->capture(want, &got);
        *out = train_tree(ds, samples, num_samples, num_classes, *config, tree_id, seed_counter,
                          CF_TRAIN_LEVEL_BATCHED, nullptr);
        CF_CUDA_CHECK(cudaStreamSynchronize(ds->ctx->stream));
        CF_REQUIRE(static_cast<int>(got.size()) <= num_levels, "cf_train_tree_snapshots: internal: too many levels");
        for (size_t i = 0; i < got.size(); i++) snapshots[i] = got[i];
        *num_snapshots = static_cast<int>(got.size());
        disarm.ok = true;
    });
}

cf_status cf_level_snapshot_info(cf_level_snapshot* s, int* level, int* num_nodes, int64_t* num_samples) {
    return guard([&] {
        CF_REQUIRE(s, "cf_level_snapshot_info: snapshot is NULL");
        if (level) *level = s->level;
        if (num_nodes) *num_nodes = s->M;
        if (num_samples) *num_samples = s->n;
    });
}

cf_status cf_level_snapshot_export(cf_level_snapshot* s, int64_t* node_offsets, cf_sample* samples, uint32_t* seed) {
    return guard([&] {
        CF_REQUIRE(s, "cf_level_snapshot_export: snapshot is NULL");
        make_current(s->ds->ctx);
        if (node_offsets) std::memcpy(node_offsets, s->offsets.data(), sizeof(int64_t) * (s->M + 1));
        if (samples)
            CF_CUDA_CHECK(cudaMemcpy(samples, s->samples.get(), sizeof(cf_sample) * s->n, cudaMemcpyDeviceToHost));
        if (seed) *seed = s->seed;
    });
}

cf_status cf_level_snapshot_run(cf_level_snapshot* s, int mode, cf_split* best, double* device_ms,
                                int64_t* feature_evals, int* next_nodes, int64_t* next_samples) {
    return guard([&] {
        CF_REQUIRE(s && s->ds && s->ds->trainer, "cf_level_snapshot_run: snapshot or its dataset is gone");
        CF_REQUIRE(mode == CF_TRAIN_LEVEL_BATCHED || mode == CF_TRAIN_PER_NODE, "cf_level_snapshot_run: unknown mode");
        static_cast<TreeTrainer*>(s->ds->trainer)->run_level(s, mode, best);
        if (device_ms) *device_ms = s->last_ms;
        if (feature_evals) *feature_evals = s->last_evals;
        if (next_nodes) *next_nodes = s->next_nodes;
        if (next_samples) *next_samples = s->next_samples;
    });
}

cf_status cf_level_snapshot_destroy(cf_level_snapshot* s) {
    return guard([&] { delete s; });
}

cf_status cf_tree_info(cf_tree* tree, int* num_nodes, int* num_classes, int* depth, int* tree_id) {
    return guard([&] {
        CF_REQUIRE(tree, "cf_tree_info: tree is NULL");
        if (num_nodes) *num_nodes = tree->num_nodes;
        if (num_classes) *num_classes = tree->C;
        if (depth) *depth = tree->depth();
        if (tree_id) *tree_id = tree->tree_id;
    });
}

cf_status cf_tree_export(cf_tree* tree, int32_t* level, int32_t* left, int8_t* feature, float* threshold, double* score,
                         int32_t* feature_id, uint32_t* histogram, uint32_t* num_samples) {
    return guard([&] {
        CF_REQUIRE(tree, "cf_tree_export: tree is NULL");
        const size_t n = tree->num_nodes;
        if (level) std::memcpy(level, tree->level.data(), 4 * n);
        if (left) std::memcpy(left, tree->left.data(), 4 * n);
        if (feature) std::memcpy(feature, tree->feature.data(), 11 * n);
        if (threshold) std::memcpy(threshold, tree->threshold.data(), 4 * n);
        if (score) std::memcpy(score, tree->score.data(), 8 * n);
        if (feature_id) std::memcpy(feature_id, tree->feature_id.data(), 4 * n);
        if (histogram) std::memcpy(histogram, tree->hist.data(), 4 * n * tree->C);
        if (num_samples) std::memcpy(num_samples, tree->nsamp.data(), 4 * n);
    });
}

cf_status cf_tree_import(int tree_id, int num_nodes, int num_classes, const int32_t* level, const int32_t* left,
                         const int8_t* feature, const float* threshold, const double* score, const int32_t* feature_id,
                         const uint32_t* histogram, cf_tree** out) {
    return guard([&] {
        CF_REQUIRE(out && left && feature && threshold && histogram, "cf_tree_import: NULL argument");
        CF_REQUIRE(num_nodes >= 1 && num_classes >= 1 && num_classes <= 256, "cf_tree_import: bad sizes");
        for (int i = 0; i < num_nodes; i++)
            CF_REQUIRE(left[i] == -1 || (left[i] > i && left[i] + 1 < num_nodes),
                       "cf_tree_import: child index out of range at node " + std::to_string(i));
        auto* t = new cf_tree();
        t->tree_id = tree_id;
        t->C = num_classes;
        t->resize(num_nodes);
        const size_t n = num_nodes;
        std::memcpy(t->left.data(), left, 4 * n);
        std::memcpy(t->feature.data(), feature, 11 * n);
        std::memcpy(t->threshold.data(), threshold, 4 * n);
        std::memcpy(t->hist.data(), histogram, 4 * n * num_classes);
        if (level) std::memcpy(t->level.data(), level, 4 * n);
        if (score) std::memcpy(t->score.data(), score, 8 * n);
        else std::fill(t->score.begin(), t->score.end(), std::nan(""));
        if (feature_id) std::memcpy(t->feature_id.data(), feature_id, 4 * n);
        else std::fill(t->feature_id.begin(), t->feature_id.end(), -1);
        for (size_t i = 0; i < n; i++) {
            uint32_t s = 0;
            for (int c = 0; c < num_classes; c++) s += histogram[i * num_classes + c];
            t->nsamp[i] = s;
        }
        if (!level) {
            std::fill(t->level.begin(), t->level.end(), 0);
            t->level[0] = 1;
            for (size_t i = 0; i < n; i++)
                if (t->left[i] >= 0) t->level[t->left[i]] = t->level[t->left[i] + 1] = t->level[i] + 1;
        }
        *out = t;
    });
}

cf_status cf_tree_destroy(cf_tree* tree) {
    return guard([&] { delete tree; });
}

cf_status cf_tree_level_stats(cf_tree* tree, int capacity, int* num_levels, int32_t* nodes, int64_t* samples,
                              float* eval_ms) {
    return guard([&] {
        CF_REQUIRE(tree && num_levels, "cf_tree_level_stats: NULL argument");
        const int n = static_cast<int>(tree->level_eval_ms.size());
        *num_levels = n;
        const int m = std::min(n, capacity);
        for (int i = 0; i < m; i++) {
            if (nodes) nodes[i] = tree->level_nodes[i];
            if (samples) samples[i] = tree->level_samples[i];
            if (eval_ms) eval_ms[i] = tree->level_eval_ms[i];
        }
    });
}

cf_status cf_tree_level_starts(cf_tree* tree, int capacity, float* start_ms) {
    return guard([&] {
        CF_REQUIRE(tree && start_ms, "cf_tree_level_starts: NULL argument");
        const int m = std::min(static_cast<int>(tree->level_start_ms.size()), capacity);
        for (int i = 0; i < m; i++) start_ms[i] = tree->level_start_ms[i];
    });
}

cf_status cf_tree_train_stats(cf_tree* tree, int64_t* feature_evals, double* device_ms, int* levels) {
    return guard([&] {
        CF_REQUIRE(tree, "cf_tree_train_stats: tree is NULL");
        if (feature_evals) *feature_evals = tree->feature_evals;
        if (device_ms) *device_ms = tree->device_ms;
        if (levels) *levels = tree->levels;
    });
}

}  // extern "C"
