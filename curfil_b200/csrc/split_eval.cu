// Split search for a tree level (kernels b, c, d).
//
// Level-batched form: every open node of the level is cut into work items (node, feature range)
// and one persistent launch drains the item queue. A CTA evaluates its item tile by tile:
//   1. stage the tile's feature parameters, sorted thresholds and threshold ranks in shared memory;
//   2. for every (sample, feature) pair compute the double response exactly as the reference does,
//      locate it among the feature's sorted thresholds (binary search on the response rounded up
//      to float, which orders identically to the reference's double compare) and increment ONE
//      shared-memory bin [feature][class][position] (a plain shared atomic, or warp-aggregated with
//      __match_any_sync); the lanes of a warp take (sample, feature) pairs of neighbouring samples
//      (sample groups) or one sample each through the tile's features;
//   3. turn the bins into cumulative counts, so left(t) = bins up to rank(t), right = node - left;
//   4. score every (feature, threshold) with the normalised information gain in double and keep
//      the near-best candidates; a final per-node reduction applies the tie rule.
// Counts never leave the SM; only the candidates of each item do.
//
// Per-node form: the reference's structure (random_tree_image_gpu.cu:1455-1720, 2137-2182):
// responses [F][N] to global memory, one block per (threshold, feature) histogramming them,
// a score kernel and a host argmax, launched node by node.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>

#include <cub/device/device_radix_sort.cuh>

#include "eval_fast.cuh"
#include "split_eval.h"

namespace cf {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kUnroll = 2;   // samples per lane and step in the sample-group mapping (4 spills and is slower)
constexpr int kStagedUnroll = 2;   // samples per lane and step in the staged-bins histogram (4 was no faster)

template <bool kAgg>
__device__ __forceinline__ void bin_increment(uint32_t* bins, int key) {
    if (kAgg) {
        const unsigned peers = __match_any_sync(kFull, key);
        const int leader = __ffs(peers) - 1;
        if (key >= 0 && static_cast<int>(threadIdx.x & 31) == leader) atomicAdd(bins + key, __popc(peers));
    } else {
        if (key >= 0) atomicAdd(bins + key, 1u);
    }
}

// Scoring constants of one node: the sample total, the classification entropy and the constants of
// the score bounds, all over the present classes in ascending label order.
struct NodeConsts {
    double total, hc;
    ScoreConsts k;
};

// One thread per node: the constants every work item of the node would otherwise compute on one
// thread (a few double logarithms per class) while the CTA waits.
__global__ void node_consts_kernel(int M, int C, const uint32_t* __restrict__ node_hist, NodeConsts* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M) return;
    uint32_t counts[256];
    int cp = 0;
    for (int c = 0; c < C; c++) {
        const uint32_t h = node_hist[static_cast<long long>(n) * C + c];
        if (h > 0) counts[cp++] = h;
    }
    double total = 0;
    for (int i = 0; i < cp; i++) total += static_cast<double>(counts[i]);
    NodeConsts r;
    r.total = total;
    r.hc = classification_entropy(cp, counts, total);
    r.k = score_consts(counts, cp);
    out[n] = r;
}

struct EvalArgs {
    DsView ds;
    const Sample* samples;
    const NodeDesc* nodes;
    const uint32_t* node_hist;
    int C, F, T;
    const FeatParams* packs;
    const float* sorted_thr;
    const uint16_t* ranks;
    const EvalItem* items;
    const int* order;
    int n_items;
    int* queue;
    ItemCandidates* cands;
    int ft_max;
    int bins_budget;
    uint32_t* group_bins;  // [groups][bins_budget] merged counts of chunked items, zero at launch
    int* group_count;      // [groups] chunks finished, zero at launch
    uint32_t* dump_left;   // optional [M][F][T][C] left counts (tests); nullptr in training
    // staged bins: the bin of row r, feature f (g = f - staged_f0) is
    // staged[((g / 32) * staged_rows + r) * 32 + g % 32]: 32-feature blocks, each [rows][32 bytes]; the
    // rows of node n start at row_base[n], and row_label holds each row's label. nullptr: the kernel
    // computes its bins itself.
    const uint8_t* staged = nullptr;
    long long staged_rows = 0;
    int staged_f0 = 0;
    const long long* row_base = nullptr;
    const uint8_t* row_label = nullptr;
    const int* staged_flip_both = nullptr;   // nonzero: a sample of the level has flip 2
    // fused search over a copy of the samples sorted by (node, frame, Morton code): node n's samples
    // are rows row_base[n] .. of it; nullptr: the level's own array
    const Sample* sorted_samples = nullptr;
    // per-node scoring constants computed once per level (node_consts_kernel); nullptr: every item
    // computes its node's constants itself
    const NodeConsts* node_consts = nullptr;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Features of one histogram tile: as many as the budget holds for `cp` classes and T + 1 bins, at most
// ft_max. With sample groups the lanes of a warp take (sample, feature) pairs in groups of a power of
// two, so the tile is rounded down to one: 5 features would keep 3 of every 8 lanes idle, 4 keep all
// 32 busy (the samples are read once more per tile, which costs far less).
__host__ __device__ inline int tile_features(int budget, int cp, int T1, int ft_max, bool grouped) {
    int ft = budget / (cp * T1);
    ft = ft < 1 ? 1 : (ft > ft_max ? ft_max : ft);
    if (grouped && ft < 32) {
        int p = 1;
        while (2 * p <= ft) p *= 2;
        ft = p;
    }
    return ft;
}

// TP = stride of a feature's threshold row (T, or 32 for the padded search)
struct SmemLayout {
    size_t counts, params, thr, rank, scores, bins, total;
    __host__ __device__ SmemLayout(int C, int T, int TP, int ft_max, int budget) {
        size_t o = 0;
        counts = o;
        o += align16(sizeof(uint32_t) * C);
        params = o;
        o += align16(sizeof(EvalFeat) * ft_max);
        thr = o;
        o += align16(sizeof(float) * ft_max * TP);
        rank = o;
        o += align16(sizeof(uint16_t) * ft_max * T);
        scores = o;
        o += align16(sizeof(double) * ft_max * T);
        bins = o;
        o += align16(sizeof(uint32_t) * budget);
        total = o;
    }
};

// Normalised information gain of one (feature, threshold) from cumulative bins.
// cum points at bins[f][0][rank]; stride between classes is T + 1.
__device__ __noinline__ double score_from_cum(const uint32_t* cum, int stride, const uint32_t* counts, int cp, double total,
                                        double hc) {
    uint32_t L = 0;
    for (int i = 0; i < cp; i++) L += cum[i * stride];
    const double Ld = static_cast<double>(L);
    const double Rd = __dsub_rn(total, Ld);
    if (L == 0 || Rd == 0.0) return 0.0;
    const double leftProb = __ddiv_rn(Ld, total);
    const double rightProb = __ddiv_rn(Rd, total);
    double ig = 0;
    for (int i = 0; i < cp; i++) {
        const uint32_t h = counts[i];
        const uint32_t l = cum[i * stride];
        const uint32_t r = h - l;
        const double classProb = __ddiv_rn(static_cast<double>(h), total);
        if (l > 0) ig = __dadd_rn(ig, ig_term(static_cast<double>(l), total, leftProb, classProb));
        if (r > 0) ig = __dadd_rn(ig, ig_term(static_cast<double>(r), total, rightProb, classProb));
    }
    ig = normalize_score(ig);
    if (ig == 0) return 0.0;
    const double hs = __ddiv_rn(__dsub_rn(__dadd_rn(entropy_of(Ld), entropy_of(Rd)), entropy_of(total)), total);
    return normalize_score(__ddiv_rn(__dmul_rn(2.0, ig), __dadd_rn(hs, hc)));
}

// score_from_cum with the work spread over a warp: the lanes evaluate the per-class terms (their
// divisions and logarithms) and the three entropies in parallel, and every lane adds the terms in
// score_from_cum's order, so the result is bit-identical (the serial form spends about 300 cycles
// of dependent double arithmetic per class on one thread while its CTA waits). Called by all lanes.
__device__ __noinline__ double score_from_cum_warp(const uint32_t* cum, int stride, const uint32_t* counts, int cp,
                                                   double total, double hc, int lane) {
    uint32_t L = 0;
    for (int i = lane; i < cp; i += 32) L += cum[i * stride];
    for (int off = 16; off > 0; off >>= 1) L += __shfl_xor_sync(kFull, L, off);
    const double Ld = static_cast<double>(L);
    const double Rd = __dsub_rn(total, Ld);
    if (L == 0 || Rd == 0.0) return 0.0;
    const double leftProb = __ddiv_rn(Ld, total);
    const double rightProb = __ddiv_rn(Rd, total);
    double e = 0.0;
    if (lane == 1) e = entropy_of(Ld);
    else if (lane == 2) e = entropy_of(Rd);
    else if (lane == 3) e = entropy_of(total);
    double ig = 0;
    for (int base = 0; base < cp; base += 32) {
        const int i = base + lane;
        double tl = 0.0, tr = 0.0;
        bool hl = false, hr = false;
        if (i < cp) {
            const uint32_t h = counts[i];
            const uint32_t l = cum[i * stride];
            const uint32_t r = h - l;
            const double classProb = __ddiv_rn(static_cast<double>(h), total);
            hl = l > 0;
            hr = r > 0;
            if (hl) tl = ig_term(static_cast<double>(l), total, leftProb, classProb);
            if (hr) tr = ig_term(static_cast<double>(r), total, rightProb, classProb);
        }
        const unsigned bl = __ballot_sync(kFull, hl), br = __ballot_sync(kFull, hr);
        const int m = min(32, cp - base);
        for (int j = 0; j < m; j++) {
            const double x = __shfl_sync(kFull, tl, j);
            const double y = __shfl_sync(kFull, tr, j);
            if ((bl >> j) & 1u) ig = __dadd_rn(ig, x);
            if ((br >> j) & 1u) ig = __dadd_rn(ig, y);
        }
    }
    ig = normalize_score(ig);   // the same value on every lane
    if (ig == 0) return 0.0;
    const double eL = __shfl_sync(kFull, e, 1), eR = __shfl_sync(kFull, e, 2), eT = __shfl_sync(kFull, e, 3);
    const double hs = __ddiv_rn(__dsub_rn(__dadd_rn(eL, eR), eT), total);
    return normalize_score(__ddiv_rn(__dmul_rn(2.0, ig), __dadd_rn(hs, hc)));
}

constexpr int kExactList = 256;   // pairs of a tile listed for the exact score (more: scored where found)

template <bool kAgg, int kPad, int kMinBlocks, bool kGrouped>
__global__ void __launch_bounds__(256, kMinBlocks)
level_eval_kernel(EvalArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_item;
    __shared__ uint8_t s_lid[256];
    __shared__ uint8_t s_pc[256];   // dense class id -> label
    __shared__ int s_warp_cnt[8];
    __shared__ int s_cp;
    __shared__ double s_total, s_hc;
    __shared__ ScoreConsts s_k;
    __shared__ float s_wmax[8];
    __shared__ double s_best;
    __shared__ double s_cs[kMaxCand];
    __shared__ int s_ct[kMaxCand], s_cf[kMaxCand];
    __shared__ int s_exact[kExactList];   // a tile's pairs needing the exact score
    __shared__ int s_nexact;
    __shared__ double s_ns[kMaxCand];   // a tile's new candidates
    __shared__ int s_nt[kMaxCand], s_nf[kMaxCand];
    __shared__ int s_cn;
    __shared__ double s_drop;
    __shared__ int s_last;

    const int TP = kPad ? kPad : a.T;
    // threshold row stride in shared memory: with sample groups the lanes of a warp search different
    // features' rows at the same position, so the rows are skewed by one bank
    const int TPS = TP + (kGrouped ? 1 : 0);
    const SmemLayout L(a.C, a.T, TP + 1, a.ft_max, a.bins_budget);
    uint32_t* s_counts = reinterpret_cast<uint32_t*>(smem + L.counts);
    EvalFeat* s_params = reinterpret_cast<EvalFeat*>(smem + L.params);
    float* s_thr = reinterpret_cast<float*>(smem + L.thr);
    uint16_t* s_rank = reinterpret_cast<uint16_t*>(smem + L.rank);
    double* s_scores = reinterpret_cast<double*>(smem + L.scores);
    uint32_t* s_bins = reinterpret_cast<uint32_t*>(smem + L.bins);

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int T = a.T;
    const int T1 = T + 1;

    for (;;) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(a.queue, 1);
        __syncthreads();
        const int q = s_item;
        if (q >= a.n_items) return;
        const int item_id = a.order[q];
        const EvalItem item = a.items[item_id];
        const NodeDesc nd = a.nodes[item.node];
        const uint32_t* hist = a.node_hist + static_cast<long long>(item.node) * a.C;

        // ---- class compaction: present classes get dense ids in ascending label order
        {
            const uint32_t cnt = tid < a.C ? hist[tid] : 0u;
            const bool present = cnt > 0;
            const unsigned bal = __ballot_sync(kFull, present);
            if (lane == 0) s_warp_cnt[warp] = __popc(bal);
            __syncthreads();
            int base = 0;
            for (int w = 0; w < warp; w++) base += s_warp_cnt[w];
            const int idx = base + __popc(bal & ((1u << lane) - 1u));
            if (tid < 256) s_lid[tid] = present ? static_cast<uint8_t>(idx) : static_cast<uint8_t>(255);
            if (present) s_pc[idx] = static_cast<uint8_t>(tid);
            if (present) s_counts[idx] = cnt;
            if (tid == 0) {
                int cp = 0;
                for (int w = 0; w < 8; w++) cp += s_warp_cnt[w];
                s_cp = cp;
                s_best = -INFINITY;
                s_cn = 0;
                s_drop = -INFINITY;
                if (a.node_consts) {
                    const NodeConsts nc = a.node_consts[item.node];
                    s_total = nc.total;
                    s_hc = nc.hc;
                    s_k = nc.k;
                }
            }
            __syncthreads();
            if (!a.node_consts) {
                if (tid == 0) {
                    // node total and classification entropy, classes in ascending label order (score.h:174-189)
                    double total = 0;
                    for (int i = 0; i < s_cp; i++) total += static_cast<double>(s_counts[i]);
                    s_total = total;
                    s_hc = classification_entropy(s_cp, s_counts, total);
                    s_k = score_consts(s_counts, s_cp);
                }
                __syncthreads();
            }
        }
        const ScoreConsts sk = s_k;
        const int cp = s_cp;
        const double total = s_total;
        const double hc = s_hc;
        // the item's samples: the whole node, or one chunk of it
        const bool chunked = item.chunks > 1;
        const int N = chunked ? item.s_end - item.s_begin : nd.count;
        // the node's samples in the level's order, or in the Morton-sorted copy (rows node by node)
        const Sample* const smps = a.sorted_samples ? a.sorted_samples : a.samples;
        const long long sbase = (a.sorted_samples ? a.row_base[item.node] : nd.start) + (chunked ? item.s_begin : 0);
        // (staged bins: a power of two <= 32 as well, so a tile never crosses a 32-feature block)
        const int ft = tile_features(a.bins_budget, cp, T1, a.ft_max, kGrouped || a.staged);

        for (int f0 = item.f_begin; f0 < item.f_end; f0 += ft) {
            const int nf = min(ft, item.f_end - f0);
            // ---- stage the tile (the parameters and thresholds only where responses are computed: not
            // for staged bins unless a sample of the level is evaluated both ways)
            const bool need_thr = !a.staged || *a.staged_flip_both;
            for (int i = tid; i < nf && need_thr; i += blockDim.x) s_params[i] = make_eval_feat(a.packs[f0 + i]);
            const float* g_thr = a.sorted_thr + static_cast<long long>(f0) * T;
            if (!need_thr) {
            } else if (kPad) {
                constexpr int kShift = kPad == 64 ? 6 : 5;
                for (int i = tid; i < nf * kPad; i += blockDim.x) {
                    const int t = i & (kPad - 1);
                    s_thr[(i >> kShift) * TPS + t] = t < T ? g_thr[(i >> kShift) * T + t] : INFINITY;
                }
            } else {
                for (int i = tid; i < nf * T; i += blockDim.x) s_thr[(i / T) * TPS + i % T] = g_thr[i];
            }
            for (int i = tid; i < nf * T; i += blockDim.x) s_rank[i] = a.ranks[static_cast<long long>(f0) * T + i];
            const int nbins = nf * cp * T1;
            for (int i = tid; i < nbins; i += blockDim.x) s_bins[i] = 0u;
            __syncthreads();

            const int W = a.ds.width, H = a.ds.height;
            const int nthr = blockDim.x;
            const int n_major = kGrouped || a.staged ? 0 : (N / nthr) * nthr;
            if (a.staged) {
                // ---- histogram of staged bins: the tile (a power of two of features, so within one
                // 32-feature block) is, per sample, nw 4-byte words of the sample's 32-byte segment of
                // the block (starting `lead` bytes into the first); the node's rows are consecutive
                // segments, so a tile reads one contiguous run. WL lanes (nw rounded up to a power of
                // two) take one sample, a lane one word, i.e. four bins, and each lane kStagedUnroll
                // samples per step so that several loads are in flight. A sample evaluated both ways
                // (flip 2) has its unflipped bin staged; the flipped one is computed here by the
                // sample's first lane.
                const int off = f0 - a.staged_f0;
                const int o = off & 31;
                const int lead = o & 3;
                const int nw = (lead + nf + 3) >> 2;
                const int WL = nw <= 1 ? 1 : 1 << (32 - __clz(nw - 1));
                const int wi = lane & (WL - 1);
                const int js = lane / WL;
                const int step = static_cast<int>(blockDim.x >> 5) * (32 / WL);
                const long long row0 = a.row_base[item.node] + (sbase - nd.start);
                const uint8_t* rows = a.staged + ((static_cast<long long>(off >> 5) * a.staged_rows + row0) << 5) + (o - lead);
                for (int s0 = warp * (32 / WL); s0 < N; s0 += kStagedUnroll * step) {   // trip count uniform in a warp
                    uint32_t v[kStagedUnroll];
                    int lid[kStagedUnroll], flip[kStagedUnroll];
                    bool act[kStagedUnroll];
                    Sample smp[kStagedUnroll];
#pragma unroll
                    for (int u = 0; u < kStagedUnroll; u++) {
                        const int s = s0 + js + u * step;
                        const bool sv = s < N;
                        const int sc = sv ? s : N - 1;
                        act[u] = sv && wi < nw;
                        v[u] = act[u] ? __ldg(reinterpret_cast<const uint32_t*>(rows + (static_cast<long long>(sc) << 5)) + wi)
                                      : 0u;
                        if (need_thr) {   // a sample of the level has flip 2: the whole sample
                            smp[u] = a.samples[sbase + sc];
                            lid[u] = smp[u].label;
                            flip[u] = sv && wi == 0 ? smp[u].flip : 0;
                        } else {
                            lid[u] = a.row_label[row0 + sc];
                            flip[u] = 0;
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kStagedUnroll; u++) {
                        lid[u] = s_lid[lid[u]];
#pragma unroll
                        for (int b = 0; b < 4; b++) {
                            const int f = 4 * wi + b - lead;
                            const bool ok = act[u] && f >= 0 && f < nf;
                            bin_increment<kAgg>(s_bins,
                                                ok ? (f * cp + lid[u]) * T1 + static_cast<int>((v[u] >> (8 * b)) & 0xffu) : -1);
                        }
                    }
                    bool both = false;
#pragma unroll
                    for (int u = 0; u < kStagedUnroll; u++) both = both || flip[u] == 2;
                    if (__any_sync(kFull, both)) {
#pragma unroll
                        for (int u = 0; u < kStagedUnroll; u++) {
                            const EvalPixel px = make_eval_pixel(a.ds, smp[u]);
                            for (int f = 0; f < nf; f++) {
                                const SortedBins<kPad> sorted{s_thr + f * TPS, T};
                                const int key = flip[u] == 2
                                                    ? (f * cp + lid[u]) * T1 + feature_bin(px, W, H, s_params[f], true, sorted)
                                                    : -1;
                                bin_increment<kAgg>(s_bins, key);
                            }
                        }
                    }
                }
            } else if constexpr (kGrouped) {
                // ---- histogram, sample groups: the lanes of a warp take (sample, feature) pairs of a
                // few consecutive samples (FL lanes per sample, FL = nf rounded up to a power of two,
                // at most 32) and the warps of the CTA the next groups. The samples in flight on an SM
                // are then neighbours in the node's order, close together in the image, and the
                // corner gathers of their features share L1 lines.
                const int FL = nf >= 32 ? 32 : (nf <= 1 ? 1 : 1 << (32 - __clz(nf - 1)));
                const int SPW = 32 / FL;
                const int fl = lane & (FL - 1);
                const int js = lane / FL;
                const int step = static_cast<int>(blockDim.x >> 5) * SPW;
                if (nf <= 32) {
                    // every lane keeps one feature for all its samples: parameters in registers
                    const bool fa = fl < nf;
                    const int fc = fa ? fl : 0;
                    const EvalFeat ef = s_params[fc];
                    const SortedBins<kPad> sorted{s_thr + fc * TPS, T};
                    // kUnroll samples per lane and step: their gathers are independent and overlap
                    for (int s0 = warp * SPW; s0 < N; s0 += kUnroll * step) {   // trip count uniform in a warp
                        EvalPixel px[kUnroll];
                        int row[kUnroll], flip[kUnroll], key[kUnroll];
                        bool act[kUnroll];
#pragma unroll
                        for (int u = 0; u < kUnroll; u++) {
                            const int s = s0 + js + u * step;
                            act[u] = fa && s < N;
                            const Sample m = smps[sbase + min(s, N - 1)];
                            px[u] = make_eval_pixel(a.ds, m);
                            row[u] = (fc * cp + s_lid[m.label]) * T1;
                            flip[u] = act[u] ? m.flip : 0;
                        }
#pragma unroll
                        for (int u = 0; u < kUnroll; u++)
                            key[u] = act[u] ? row[u] + feature_bin(px[u], W, H, ef, flip[u] == 1, sorted) : -1;
#pragma unroll
                        for (int u = 0; u < kUnroll; u++) bin_increment<kAgg>(s_bins, key[u]);
                        bool both = false;
#pragma unroll
                        for (int u = 0; u < kUnroll; u++) both = both || flip[u] == 2;
                        if (__any_sync(kFull, both)) {
#pragma unroll
                            for (int u = 0; u < kUnroll; u++)
                                key[u] = flip[u] == 2 ? row[u] + feature_bin(px[u], W, H, ef, true, sorted) : -1;
#pragma unroll
                            for (int u = 0; u < kUnroll; u++) bin_increment<kAgg>(s_bins, key[u]);
                        }
                    }
                } else {
                    for (int s0 = warp * SPW; s0 < N; s0 += step) {
                        const int s = s0 + js;
                        const bool sv = s < N;
                        const Sample smp = smps[sbase + min(s, N - 1)];
                        const EvalPixel px = make_eval_pixel(a.ds, smp);
                        const int lid = s_lid[smp.label];
                        const int flip = smp.flip;
                        const bool any_both = __any_sync(kFull, sv && flip == 2);
                        for (int fb = 0; fb < nf; fb += FL) {
                            const int f = fb + fl;
                            const bool act = sv && f < nf;
                            const int fc = act ? f : 0;
                            const SortedBins<kPad> sorted{s_thr + fc * TPS, T};
                            const int row = (fc * cp + lid) * T1;
                            const int key1 = act ? row + feature_bin(px, W, H, s_params[fc], flip == 1, sorted) : -1;
                            bin_increment<kAgg>(s_bins, key1);
                            if (any_both) {
                                const int key2 =
                                    act && flip == 2 ? row + feature_bin(px, W, H, s_params[fc], true, sorted) : -1;
                                bin_increment<kAgg>(s_bins, key2);
                            }
                        }
                    }
                }
            }
            // ---- histogram, sample-major over whole blocks of samples: each thread keeps one sample
            // and walks the tile's features, so the sample's neighbourhood is reused from L1
            for (int s0 = 0; s0 < n_major; s0 += nthr) {
                const Sample smp = smps[sbase + s0 + tid];
                const EvalPixel px = make_eval_pixel(a.ds, smp);
                const int lid = s_lid[smp.label];
                const int flip = smp.flip;
                const bool any_both = __any_sync(kFull, flip == 2);
                // two features per step: their evaluations are independent, so their gathers and
                // arithmetic overlap before the two warp-synchronous increments
                int f = 0;
                for (; f + 1 < nf; f += 2) {
                    const EvalFeat& fa = s_params[f];
                    const EvalFeat& fb = s_params[f + 1];
                    const SortedBins<kPad> sa{s_thr + f * TPS, T};
                    const SortedBins<kPad> sb{s_thr + (f + 1) * TPS, T};
                    const int row_a = (f * cp + lid) * T1;
                    const int row_b = row_a + cp * T1;
                    const int ka = row_a + feature_bin(px, W, H, fa, flip == 1, sa);
                    const int kb = row_b + feature_bin(px, W, H, fb, flip == 1, sb);
                    bin_increment<kAgg>(s_bins, ka);
                    bin_increment<kAgg>(s_bins, kb);
                    if (any_both) {
                        const int ka2 = flip == 2 ? row_a + feature_bin(px, W, H, fa, true, sa) : -1;
                        const int kb2 = flip == 2 ? row_b + feature_bin(px, W, H, fb, true, sb) : -1;
                        bin_increment<kAgg>(s_bins, ka2);
                        bin_increment<kAgg>(s_bins, kb2);
                    }
                }
                if (f < nf) {
                    const EvalFeat& fp = s_params[f];
                    const SortedBins<kPad> sorted{s_thr + f * TPS, T};
                    const int row = (f * cp + lid) * T1;
                    const int key1 = row + feature_bin(px, W, H, fp, flip == 1, sorted);
                    bin_increment<kAgg>(s_bins, key1);
                    if (any_both) {
                        const int key2 = flip == 2 ? row + feature_bin(px, W, H, fp, true, sorted) : -1;
                        bin_increment<kAgg>(s_bins, key2);
                    }
                }
            }
            // ---- the remaining Nt < blockDim samples, pair-major: pairs p = f * Nt + s spread over
            // all threads with a uniform trip count so warps stay converged
            const int Nt = a.staged ? 0 : N - n_major;
            if (!kGrouped && Nt > 0) {
                const Sample* tail = smps + sbase + n_major;
                const long long pairs = static_cast<long long>(nf) * Nt;
                const int iters = static_cast<int>((pairs + nthr - 1) / nthr);
                const int qstep = nthr / Nt;
                const int rstep = nthr - qstep * Nt;
                int f = tid / Nt;
                int s = tid - f * Nt;
                for (int it = 0; it < iters; it++) {
                    int key1 = -1, key2 = -1;
                    if (f < nf) {
                        const Sample smp = tail[s];
                        const EvalPixel px = make_eval_pixel(a.ds, smp);
                        const EvalFeat& fp = s_params[f];
                        const SortedBins<kPad> sorted{s_thr + f * TPS, T};
                        const int row = (f * cp + s_lid[smp.label]) * T1;
                        key1 = row + feature_bin(px, W, H, fp, smp.flip == 1, sorted);
                        if (smp.flip == 2) key2 = row + feature_bin(px, W, H, fp, true, sorted);
                    }
                    bin_increment<kAgg>(s_bins, key1);
                    if (__any_sync(kFull, key2 >= 0)) bin_increment<kAgg>(s_bins, key2);
                    s += rstep;
                    f += qstep;
                    if (s >= Nt) {
                        s -= Nt;
                        f++;
                    }
                }
            }
            __syncthreads();

            if (chunked) {
                // ---- one chunk of the node's samples (the item is a single tile): add its counts to
                // the group's histogram in global memory and count the chunk in; the chunk that
                // arrives last loads the merged counts and scores them, the others leave the item with
                // no candidates. Integer sums, so the merged counts do not depend on the order.
                uint32_t* g = a.group_bins + static_cast<long long>(item.group) * a.bins_budget;
                for (int i = tid; i < nbins; i += blockDim.x) {
                    const uint32_t v = s_bins[i];
                    if (v) atomicAdd(g + i, v);
                }
                __threadfence();
                __syncthreads();
                if (tid == 0) s_last = atomicAdd(a.group_count + item.group, 1) == item.chunks - 1 ? 1 : 0;
                __syncthreads();
                if (!s_last) break;
                __threadfence();
                for (int i = tid; i < nbins; i += blockDim.x) s_bins[i] = __ldcg(g + i);
                __syncthreads();
            }

            // ---- cumulative counts along the threshold positions: a thread per row, or where the
            // tile has few rows (few classes present) a warp per row, 32 positions per shuffle scan
            if (nf * cp > 128) {
                for (int row = tid; row < nf * cp; row += blockDim.x) {
                    uint32_t acc = 0;
                    uint32_t* b = s_bins + row * T1;
                    for (int k = 0; k < T1; k++) {
                        acc += b[k];
                        b[k] = acc;
                    }
                }
            } else {
                for (int row = warp; row < nf * cp; row += static_cast<int>(blockDim.x >> 5)) {
                    uint32_t* b = s_bins + row * T1;
                    uint32_t carry = 0;
                    for (int k0 = 0; k0 < T1; k0 += 32) {
                        const int k = k0 + lane;
                        uint32_t v = k < T1 ? b[k] : 0u;
                        for (int o = 1; o < 32; o <<= 1) {
                            const uint32_t u = __shfl_up_sync(kFull, v, o);
                            if (lane >= o) v += u;
                        }
                        v += carry;
                        if (k < T1) b[k] = v;
                        carry = __shfl_sync(kFull, v, 31);
                    }
                }
            }
            __syncthreads();

            if (a.dump_left) {
                // test hook: left counts of every (feature, threshold, class) of the tile
                const int n = nf * T * cp;
                for (int i = tid; i < n; i += blockDim.x) {
                    const int fl = i / (T * cp);
                    const int rem = i - fl * T * cp;
                    const int t = rem / cp;
                    const int lid = rem - t * cp;
                    const uint32_t v = s_bins[(fl * cp + lid) * T1 + s_rank[fl * T + t]];
                    a.dump_left[((static_cast<long long>(item.node) * a.F + f0 + fl) * T + t) * a.C + s_pc[lid]] = v;
                }
            }

            // ---- scores of the tile: float bounds for every (feature, threshold) first; the exact
            // double score only where the upper bound reaches the 1e-13 window below the best lower
            // bound (or the item's best so far). A pair left out cannot be within the window of the
            // final best, so the candidates and the chosen split are those of scoring every pair.
            {
                float2* s_bounds = reinterpret_cast<float2*>(s_scores);   // slot i: (lb, ub), then the score
                float lbmax = 0.0f;
                for (int i = tid; i < nf * T; i += blockDim.x) {
                    const int fl = i / T;
                    const int t = i - fl * T;
                    const uint32_t* cum = s_bins + fl * cp * T1 + s_rank[fl * T + t];
                    const float2 b = score_bounds([&](int c) { return cum[c * T1]; }, s_counts, cp, sk);
                    s_bounds[i] = b;
                    lbmax = fmaxf(lbmax, b.x);
                }
                for (int off = 16; off > 0; off >>= 1) lbmax = fmaxf(lbmax, __shfl_xor_sync(kFull, lbmax, off));
                if (lane == 0) s_wmax[warp] = lbmax;
                if (tid == 0) s_nexact = 0;
                __syncthreads();
                float m = s_wmax[0];
                for (int w = 1; w < static_cast<int>(blockDim.x >> 5); w++) m = fmaxf(m, s_wmax[w]);
                const double floor_s = fmax(static_cast<double>(m), s_best) - 1e-13;
                // pairs reaching the floor: scored where found (fused search: the scoring overlaps the
                // other warps' gathers) or, reading staged bins, listed and scored after one barrier, a
                // warp each if there are few (latency) or a thread each (throughput); the rest get -inf
                const bool listed = a.staged != nullptr;
                for (int i = tid; i < nf * T; i += blockDim.x) {
                    const float ub = s_bounds[i].y;
                    double sc = -INFINITY;
                    if (static_cast<double>(ub) >= floor_s) {
                        const int k = listed ? atomicAdd(&s_nexact, 1) : kExactList;
                        if (k < kExactList) {
                            s_exact[k] = i;
                            continue;
                        }
                        const int fl = i / T;
                        const int t = i - fl * T;
                        sc = score_from_cum(s_bins + fl * cp * T1 + s_rank[fl * T + t], T1, s_counts, cp, total, hc);
                    }
                    s_scores[i] = sc;
                }
                if (listed) __syncthreads();
                const int ne = listed ? min(s_nexact, kExactList) : 0;
                const int nwarps = static_cast<int>(blockDim.x >> 5);
                if (ne <= nwarps) {
                    if (warp < ne) {
                        const int i = s_exact[warp];
                        const int fl = i / T;
                        const int t = i - fl * T;
                        const double sc = score_from_cum_warp(s_bins + fl * cp * T1 + s_rank[fl * T + t], T1, s_counts,
                                                              cp, total, hc, lane);
                        if (lane == 0) s_scores[i] = sc;
                    }
                } else {
                    for (int k = tid; k < ne; k += blockDim.x) {
                        const int i = s_exact[k];
                        const int fl = i / T;
                        const int t = i - fl * T;
                        s_scores[i] =
                            score_from_cum(s_bins + fl * cp * T1 + s_rank[fl * T + t], T1, s_counts, cp, total, hc);
                    }
                }
            }
            __syncthreads();

            // ---- near-best candidates (warp 0): window rule best - s < 1e-13, lowest (t, f) first
            if (warp == 0) {
                const int n = nf * T;
                double m = -INFINITY;
                for (int i = lane; i < n; i += 32) m = fmax(m, s_scores[i]);
                for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(kFull, m, off));
                const double mnew = fmax(m, s_best);
                if (lane == 0) {
                    int k = 0;
                    for (int j = 0; j < s_cn; j++) {
                        if (__dsub_rn(mnew, s_cs[j]) < 1e-13) {
                            s_cs[k] = s_cs[j];
                            s_ct[k] = s_ct[j];
                            s_cf[k] = s_cf[j];
                            k++;
                        }
                    }
                    s_cn = k;
                    s_best = mnew;
                }
                __syncwarp();
                // the tile's pairs inside the window in key order (threshold, then feature), all lanes
                // at once: the first kMaxCand are merged into the list, the others only raise the
                // dropped score (a tile of tied scores is kMaxCand insertions, not n)
                int taken = 0;
                double dmax = -INFINITY;
                for (int base = 0; base < n; base += 32) {
                    const int p = base + lane;
                    const int t = p / nf;
                    const int fl = p - t * nf;
                    const double sc = p < n ? s_scores[fl * T + t] : -INFINITY;
                    const bool e = p < n && __dsub_rn(mnew, sc) < 1e-13;
                    const unsigned bal = __ballot_sync(kFull, e);
                    const int rank = taken + __popc(bal & ((1u << lane) - 1u));
                    if (e && rank < kMaxCand) {
                        s_ns[rank] = sc;
                        s_nt[rank] = t;
                        s_nf[rank] = f0 + fl;
                    } else if (e) {
                        dmax = fmax(dmax, sc);
                    }
                    taken = min(kMaxCand, taken + __popc(bal));
                }
                for (int off = 16; off > 0; off >>= 1) dmax = fmax(dmax, __shfl_xor_sync(kFull, dmax, off));
                __syncwarp();
                if (lane == 0) {
                    s_drop = fmax(s_drop, dmax);
                    for (int q = 0; q < taken; q++) {
                        const int t = s_nt[q];
                        const int fg = s_nf[q];
                        const long long key = static_cast<long long>(t) * a.F + fg;
                        int pos = s_cn;
                        while (pos > 0 && static_cast<long long>(s_ct[pos - 1]) * a.F + s_cf[pos - 1] > key) pos--;
                        if (pos >= kMaxCand) {
                            s_drop = fmax(s_drop, s_ns[q]);
                            continue;
                        }
                        if (s_cn == kMaxCand) s_drop = fmax(s_drop, s_cs[kMaxCand - 1]);
                        const int last = min(s_cn, kMaxCand - 1);
                        for (int j = last; j > pos; j--) {
                            s_cs[j] = s_cs[j - 1];
                            s_ct[j] = s_ct[j - 1];
                            s_cf[j] = s_cf[j - 1];
                        }
                        s_cs[pos] = s_ns[q];
                        s_ct[pos] = t;
                        s_cf[pos] = fg;
                        s_cn = min(s_cn + 1, kMaxCand);
                    }
                }
                __syncwarp();
            }
            // no barrier here: the other warps stage the next tile while warp 0 merges the candidates
            // (it reads only the scores and the candidate list, which the next tile writes after its
            // first barrier)
        }

        if (tid == 0) {
            ItemCandidates c;
            c.best = s_best;
            c.n = s_cn;
            c.pad = 0;
            c.dropped = s_drop;
            for (int j = 0; j < kMaxCand; j++) {
                c.s[j] = j < s_cn ? s_cs[j] : -INFINITY;
                c.t[j] = j < s_cn ? s_ct[j] : 0;
                c.f[j] = j < s_cn ? s_cf[j] : 0;
            }
            a.cands[item_id] = c;
        }
    }
}

// features per pass-1 work item: two tiles (64 features) were 1 % faster than one, the samples'
// neighbourhoods serving more features while they are in L1
constexpr int kStageItemFeatures = 2 * kStageTile;

// bits 0..15 of v spread to the even bit positions (Morton order)
__device__ __forceinline__ unsigned long long spread_bits(uint32_t v) {
    unsigned long long x = v & 0xFFFFu;
    x = (x | (x << 8)) & 0x00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0Full;
    x = (x | (x << 2)) & 0x33333333ull;
    x = (x | (x << 1)) & 0x55555555ull;
    return x;
}

// ---- staged bins, pass 1 -------------------------------------------------------------------------
// Rows of the staged table: row_base[n] + k is sample k of node n. stage_rows_kernel gives every row
// its sample's position in the level's array and its pixel as the sort key of the pass-1 order: frame
// by frame, and within a frame in Morton (Z) order of (y, x), so the samples a CTA takes lie in a
// compact patch and their neighbourhoods overlap in L1 (9 % faster than raster order, whose 256
// samples span the frame's width).
__global__ void stage_rows_kernel(const NodeDesc* __restrict__ nodes, const long long* __restrict__ row_base, int M,
                                  long long rows, const Sample* __restrict__ samples, int node_shift,
                                  int* __restrict__ row_pos, uint8_t* __restrict__ row_label, unsigned long long* __restrict__ pixel_key,
                                  int* __restrict__ row_ids, int* __restrict__ flip_both) {
    const long long r = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (r >= rows) return;
    int lo = 0, hi = M - 1;   // the last node n with row_base[n] <= r
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (row_base[mid] <= r) lo = mid;
        else hi = mid - 1;
    }
    const long long p = nodes[lo].start + (r - row_base[lo]);
    const Sample s = samples[p];
    row_pos[r] = static_cast<int>(p);
    row_label[r] = s.label;
    pixel_key[r] = (static_cast<unsigned long long>(s.image) << 32) | (spread_bits(s.y) << 1) | spread_bits(s.x) |
                   (node_shift > 0 ? static_cast<unsigned long long>(lo) << node_shift : 0ull);
    row_ids[r] = static_cast<int>(r);
    if (s.flip == 2) *flip_both = 1;
}

// The Morton-sorted copy of a level's samples: out[k] is the sample of the k-th row in key order.
__global__ void gather_sorted_samples_kernel(long long rows, const int* __restrict__ order, const int* __restrict__ row_pos,
                                             const Sample* __restrict__ samples, Sample* __restrict__ out) {
    const long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (k < rows) out[k] = samples[row_pos[order[k]]];
}

struct StageArgs {
    DsView ds;
    const Sample* samples;
    const int* frame_order;   // [rows] rows sorted by frame (stable)
    const int* row_pos;       // [rows] sample position of each row
    long long rows;
    const FeatParams* packs;
    const float* sorted_thr;  // [F][T]
    int T;
    int f_first, n_feat;      // this chunk's features [f_first, f_first + n_feat)
    uint8_t* out;             // [n_feat / 32 blocks][rows][32]
};

// One work item = 256 consecutive rows of the frame order x one tile of kStageTile features; items are
// taken row-block-major, so the resident CTAs evaluate the samples of one or two frames at a time and
// their corner gathers hit L2. A thread takes one sample through the tile's features (two at a time,
// their gathers overlapping) and stores each four bins as one word of its row. The bin is that of the
// fused kernel's feature_bin: the unflipped response for flip 0 and 2, the flipped one for flip 1.
constexpr int kStageCtasPerSm = 3;   // 4 (56 registers fit) was 5-7 % slower: less L1 per CTA

template <int kPad>
__global__ void __launch_bounds__(256, kStageCtasPerSm)
stage_bins_kernel(StageArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    EvalFeat* s_params = reinterpret_cast<EvalFeat*>(smem);
    float* s_thr = reinterpret_cast<float*>(smem + sizeof(EvalFeat) * kStageItemFeatures);
    const int T = a.T;
    const int TP = kPad ? kPad : T;
    // (rows padded against the two-way bank conflicts of the search, one word after every 32, were
    // 2 % slower: the conflicts cost less than the extra index arithmetic)
    const int TPS = TP;
    const int W = a.ds.width, H = a.ds.height;
    const int tiles = (a.n_feat + kStageItemFeatures - 1) / kStageItemFeatures;
    const long long blocks = (a.rows + 255) / 256;
    const long long n_items = blocks * tiles;
    for (long long q = blockIdx.x; q < n_items; q += gridDim.x) {
        const long long blk = q / tiles;
        const int j = static_cast<int>(q - blk * tiles);
        const int fb = j * kStageItemFeatures;
        const int nf = min(kStageItemFeatures, a.n_feat - fb);
        const int fg = a.f_first + fb;
        __syncthreads();   // the previous item's reads of the tile are done
        for (int i = threadIdx.x; i < nf; i += blockDim.x) s_params[i] = make_eval_feat(a.packs[fg + i]);
        const float* g_thr = a.sorted_thr + static_cast<long long>(fg) * T;
        for (int i = threadIdx.x; i < nf * TP; i += blockDim.x) {
            const int f = i / TP, t = i - f * TP;
            s_thr[f * TPS + t] = t < T ? g_thr[f * T + t] : INFINITY;
        }
        __syncthreads();
        const long long r = blk * 256 + threadIdx.x;
        if (r < a.rows) {
            const int row = a.frame_order[r];
            const Sample smp = a.samples[a.row_pos[row]];
            const EvalPixel px = make_eval_pixel(a.ds, smp);
            const bool flip = smp.flip == 1;
            uint8_t* seg = a.out + (static_cast<long long>(row) << 5);   // the row's segment of block 0
            uint32_t acc = 0;
            for (int f = 0; f < nf; f += 2) {
                const int b0 = feature_bin(px, W, H, s_params[f], flip, SortedBins<kPad>{s_thr + f * TPS, T});
                const int b1 =
                    f + 1 < nf ? feature_bin(px, W, H, s_params[f + 1], flip, SortedBins<kPad>{s_thr + (f + 1) * TPS, T}) : 0;
                acc |= static_cast<uint32_t>(b0 | (b1 << 8)) << (8 * (f & 3));
                if ((f & 3) == 2 || f + 2 >= nf) {
                    const int fw = fb + (f & ~3);   // first feature of the word
                    *reinterpret_cast<uint32_t*>(seg + ((static_cast<long long>(fw >> 5) * a.rows) << 5) + (fw & 31)) = acc;
                    acc = 0;
                }
            }
        }
    }
}

// One warp per node: the global tie rule over the candidates of the node's items. The lanes stride
// over the items; the best score is a max-reduction and the chosen candidate the lowest (threshold,
// feature) key within the 1e-13 window, a min-reduction, so the result does not depend on how the
// items are spread over the lanes. (The top levels' sliced nodes have up to ~10^5 items.)
__global__ void reduce_candidates_kernel(int M, int F, const int* __restrict__ item_range,
                                         const ItemCandidates* __restrict__ cands, const float* __restrict__ thr,
                                         cf_split* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int node = static_cast<int>((blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5);
    if (node >= M) return;   // uniform per warp
    const int b = item_range[node], e = item_range[node + 1];
    double m = -INFINITY;
    for (int i = b + lane; i < e; i += 32) m = fmax(m, cands[i].best);
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(kFull, m, off));
    int ovf = 0;
    long long best_key = LLONG_MAX;
    double best_s = m;
    for (int i = b + lane; i < e; i += 32) {
        const ItemCandidates& c = cands[i];
        ovf |= __dsub_rn(m, c.dropped) < 1e-13 ? 1 : 0;
        for (int j = 0; j < c.n; j++) {
            if (__dsub_rn(m, c.s[j]) < 1e-13) {
                const long long key = static_cast<long long>(c.t[j]) * F + c.f[j];
                if (key < best_key) {
                    best_key = key;
                    best_s = c.s[j];
                }
            }
        }
    }
    ovf = __any_sync(kFull, ovf) ? 1 : 0;
    for (int off = 16; off > 0; off >>= 1) {
        const long long k2 = __shfl_xor_sync(kFull, best_key, off);
        const double s2 = __shfl_xor_sync(kFull, best_s, off);
        if (k2 < best_key) {
            best_key = k2;
            best_s = s2;
        }
    }
    if (lane != 0) return;
    const int bt = best_key == LLONG_MAX ? 0 : static_cast<int>(best_key / F);
    const int bf = best_key == LLONG_MAX ? 0 : static_cast<int>(best_key - static_cast<long long>(bt) * F);
    cf_split r;
    r.score = best_s;
    r.feature = bf;
    r.threshold_index = bt;
    r.threshold = thr[static_cast<long long>(bt) * F + bf];
    r.flags = ovf;
    out[node] = r;
}

// ---- reference-structured kernels --------------------------------------------------------------

// featureResponseKernel layout: block (4 samples, 32 features), responses [F][N]
__global__ void plain_response_kernel(DsView ds, const Sample* __restrict__ samples, int N, const int8_t* __restrict__ table,
                                      int F, double* __restrict__ resp1, double* __restrict__ resp2) {
    const int feature = blockIdx.x * blockDim.y + threadIdx.y;
    const int sample = blockIdx.y * blockDim.x + threadIdx.x;
    if (feature >= F || sample >= N) return;
    const FeatParams fp = load_feature(table, F, feature);
    const Sample s = samples[sample];
    const long long o = static_cast<long long>(feature) * N + sample;
    resp1[o] = sample_response(ds, s, fp, s.flip == 1);
    if (s.flip == 2 && resp2) resp2[o] = sample_response(ds, s, fp, true);
}

// aggregateHistogramsKernel structure: one block per (threshold, feature); per-label left/right
// counters in shared memory (uint32, any number of classes), added into counters [F][T][C][2].
__global__ void plain_histogram_kernel(const double* __restrict__ resp1, const double* __restrict__ resp2,
                                       const Sample* __restrict__ samples, int N, const float* __restrict__ thr, int F,
                                       int T, int C, uint32_t* __restrict__ counters) {
    extern __shared__ uint32_t s_cnt[];
    const int thresh = blockIdx.x;
    const int feature = blockIdx.y;
    const float threshold = thr[static_cast<long long>(thresh) * F + feature];
    for (int i = threadIdx.x; i < 2 * C; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    const double* r1 = resp1 + static_cast<long long>(feature) * N;
    const double* r2 = resp2 ? resp2 + static_cast<long long>(feature) * N : nullptr;
    for (int s = threadIdx.x; s < N; s += blockDim.x) {
        const Sample smp = samples[s];
        const int v = !(r1[s] <= threshold);
        atomicAdd(&s_cnt[2 * smp.label + v], 1u);
        if (smp.flip == 2) {
            const int v2 = !(r2[s] <= threshold);
            atomicAdd(&s_cnt[2 * smp.label + v2], 1u);
        }
    }
    __syncthreads();
    uint32_t* out = counters + (static_cast<long long>(feature) * T + thresh) * C * 2;
    for (int i = threadIdx.x; i < 2 * C; i += blockDim.x) out[i] += s_cnt[i];
}

// scoreKernel: one thread per (threshold, feature); scores [T][F]
// Float score bounds [T][F] from counters [F][T][C][2] (the level kernel's screening, standalone).
__global__ void score_bounds_kernel(const uint32_t* __restrict__ counters, const uint32_t* __restrict__ hist, int C,
                                    int F, int T, float* __restrict__ lower, float* __restrict__ upper) {
    __shared__ ScoreConsts s_k;
    if (threadIdx.x == 0) s_k = score_consts(hist, C);
    __syncthreads();
    const int feature = blockIdx.x * blockDim.x + threadIdx.x;
    const int thresh = blockIdx.y;
    if (feature >= F) return;
    const uint32_t* lr = counters + (static_cast<long long>(feature) * T + thresh) * C * 2;
    const float2 b = score_bounds([&](int c) { return lr[2 * c]; }, hist, C, s_k);
    lower[static_cast<long long>(thresh) * F + feature] = b.x;
    upper[static_cast<long long>(thresh) * F + feature] = b.y;
}

__global__ void plain_score_kernel(const uint32_t* __restrict__ counters, const uint32_t* __restrict__ hist, int C, int F,
                                   int T, double* __restrict__ scores) {
    __shared__ double s_hc;
    if (threadIdx.x == 0) {
        double total = 0, hc = 0;
        for (int c = 0; c < C; c++) total += static_cast<double>(hist[c]);
        for (int c = 0; c < C; c++)
            if (hist[c] > 0) hc = __dadd_rn(hc, entropy_of(static_cast<double>(hist[c])));
        hc = __dsub_rn(hc, entropy_of(total));
        s_hc = __ddiv_rn(hc, total);
    }
    __syncthreads();
    const int feature = blockIdx.x * blockDim.x + threadIdx.x;
    const int thresh = blockIdx.y;
    if (feature >= F) return;
    const uint32_t* lr = counters + (static_cast<long long>(feature) * T + thresh) * C * 2;
    double Ld = 0, Rd = 0;
    for (int c = 0; c < C; c++) {
        Ld += static_cast<double>(lr[2 * c]);
        Rd += static_cast<double>(lr[2 * c + 1]);
    }
    const double total = __dadd_rn(Ld, Rd);
    double score = 0.0;
    if (Ld != 0.0 && Rd != 0.0) {
        const double leftProb = __ddiv_rn(Ld, total);
        const double rightProb = __ddiv_rn(Rd, total);
        double ig = 0;
        for (int c = 0; c < C; c++) {
            const uint32_t l = lr[2 * c], r = lr[2 * c + 1];
            const double classProb = __ddiv_rn(static_cast<double>(hist[c]), total);
            if (l > 0) ig = __dadd_rn(ig, ig_term(static_cast<double>(l), total, leftProb, classProb));
            if (r > 0) ig = __dadd_rn(ig, ig_term(static_cast<double>(r), total, rightProb, classProb));
        }
        ig = normalize_score(ig);
        if (ig != 0) {
            const double hs =
                __ddiv_rn(__dsub_rn(__dadd_rn(entropy_of(Ld), entropy_of(Rd)), entropy_of(total)), total);
            score = normalize_score(__ddiv_rn(__dmul_rn(2.0, ig), __dadd_rn(hs, s_hc)));
        }
    }
    scores[static_cast<long long>(thresh) * F + feature] = score;
}

// Shared-memory layout of a level_eval launch; budget = histogram words (at least one feature).
SmemLayout level_eval_smem(int C, int T, const EvalTuning& tuning, int* budget) {
    *budget = std::max(tuning.bins_budget_words, C * (T + 1));
    // with sample groups a tile holds a power-of-two number of features: the budget is trimmed to the
    // largest such tile for all C classes, so no shared memory is reserved that no tile of a node
    // with every class present would use (what is left stays L1); nodes with fewer classes fit the
    // same or more features in it
    if (tuning.sample_groups) *budget = tile_features(*budget, C, T + 1, tuning.ft_max, true) * C * (T + 1);
    const int TP = padded_row(T) ? padded_row(T) : T;
    return SmemLayout(C, T, TP + 1, tuning.ft_max, *budget);   // rows skewed by one bank with sample groups
}

// Shared-memory carveout (percent of the SM's 228 KB) that just holds `ctas` CTAs of `smem` dynamic
// bytes (+ static shared memory and the 1 KB the runtime reserves per CTA); the rest of the unified
// 256 KB stays L1, which caches the integral-image gathers.
template <typename K>
void set_level_eval_smem(K kernel, size_t smem, int ctas) {
    cudaFuncAttributes fa;
    CF_CUDA_CHECK(cudaFuncGetAttributes(&fa, kernel));
    CF_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    const double need = static_cast<double>(ctas) * (smem + fa.sharedSizeBytes + 1024);
    const int pct = std::min(100, static_cast<int>(std::ceil(100.0 * need / (228.0 * 1024))));
    CF_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
}

template <bool kAgg, int kPad, bool kGrouped>
void launch_level_eval_g(cf_context* ctx, const EvalArgs& args, int grid, size_t smem, int ctas_per_sm) {
    if (ctas_per_sm >= 4) {
        set_level_eval_smem(level_eval_kernel<kAgg, kPad, 4, kGrouped>, smem, ctas_per_sm);
        launch(ctx, "level_eval", dim3(grid), dim3(256), smem, level_eval_kernel<kAgg, kPad, 4, kGrouped>, args);
    } else {
        set_level_eval_smem(level_eval_kernel<kAgg, kPad, 3, kGrouped>, smem, ctas_per_sm);
        launch(ctx, "level_eval", dim3(grid), dim3(256), smem, level_eval_kernel<kAgg, kPad, 3, kGrouped>, args);
    }
}

template <bool kAgg, int kPad>
void launch_level_eval_t(cf_context* ctx, const EvalArgs& args, int grid, size_t smem, int ctas_per_sm,
                         bool grouped) {
    if (grouped) launch_level_eval_g<kAgg, kPad, true>(ctx, args, grid, smem, ctas_per_sm);
    else launch_level_eval_g<kAgg, kPad, false>(ctx, args, grid, smem, ctas_per_sm);
}

template <bool kAgg>
void launch_level_eval_a(cf_context* ctx, const EvalArgs& args, int grid, size_t smem, int ctas_per_sm,
                         bool grouped) {
    switch (padded_row(args.T)) {
        case 32: launch_level_eval_t<kAgg, 32>(ctx, args, grid, smem, ctas_per_sm, grouped); break;
        case 64: launch_level_eval_t<kAgg, 64>(ctx, args, grid, smem, ctas_per_sm, grouped); break;
        default: launch_level_eval_t<kAgg, 0>(ctx, args, grid, smem, ctas_per_sm, grouped); break;
    }
}

template <int kPad>
void launch_stage_bins_t(cf_context* ctx, const StageArgs& a) {
    const int TP = kPad ? kPad : a.T;
    const size_t smem = sizeof(EvalFeat) * kStageItemFeatures + sizeof(float) * kStageItemFeatures * TP;
    set_level_eval_smem(stage_bins_kernel<kPad>, smem, kStageCtasPerSm);
    const long long items = (a.rows + 255) / 256 * ((a.n_feat + kStageItemFeatures - 1) / kStageItemFeatures);
    const int grid = static_cast<int>(std::min<long long>(items, static_cast<long long>(ctx->num_sms) * kStageCtasPerSm));
    launch(ctx, "stage_bins", dim3(grid), dim3(256), smem, stage_bins_kernel<kPad>, a);
}

void launch_stage_bins(cf_context* ctx, const StageArgs& a) {
    switch (padded_row(a.T)) {
        case 32: launch_stage_bins_t<32>(ctx, a); break;
        case 64: launch_stage_bins_t<64>(ctx, a); break;
        default: launch_stage_bins_t<0>(ctx, a); break;
    }
}

// The level_eval instance for the tuning and threshold count (T <= 31 and 32 <= T <= 63 take the
// padded branch-free searches).
void launch_level_eval(cf_context* ctx, const EvalArgs& args, int grid, const EvalTuning& tuning) {
    int budget = 0;
    const SmemLayout lay = level_eval_smem(args.C, args.T, tuning, &budget);
    CF_REQUIRE(lay.total + 4096 <= ctx->smem_per_block_optin,
               "split search: classes x thresholds too large for shared memory");
    CF_REQUIRE(args.bins_budget == budget && args.ft_max == tuning.ft_max, "split search: inconsistent tuning");
    const bool g = tuning.sample_groups != 0;
    if (tuning.warp_aggregate) launch_level_eval_a<true>(ctx, args, grid, lay.total, tuning.ctas_per_sm, g);
    else launch_level_eval_a<false>(ctx, args, grid, lay.total, tuning.ctas_per_sm, g);
}

}  // namespace

EvalTuning EvalTuning::of(cf_context* ctx) {
    cf_eval_tuning t;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        t = ctx->tuning;
    }
    EvalTuning e;
    e.ft_max = t.features_per_tile;
    e.bins_budget_words = t.bins_budget_words;
    e.warp_aggregate = t.warp_aggregate;
    e.ctas_per_sm = t.ctas_per_sm;
    e.items_per_slot = t.items_per_slot;
    e.feature_granule = t.feature_granule;
    e.sample_groups = t.sample_groups;
    e.min_item_evals = t.min_item_evals;
    e.stage_bins = t.stage_bins;
    e.stage_max_mb = t.stage_max_mb;
    e.sample_order = t.sample_order;
    return e;
}

void plan_level_items(const std::vector<int>& node_counts, int F, const EvalTuning& tuning, int slots,
                      std::vector<EvalItem>& items, std::vector<int>& range, std::vector<int>& order,
                      int chunk_features, int* n_groups, int max_groups) {
    const int M = static_cast<int>(node_counts.size());
    const int g = std::max(1, tuning.feature_granule);
    long long total_work = 0;
    for (int n : node_counts) total_work += static_cast<long long>(n) * F;
    // items_per_slot items per resident CTA, or fewer where that would make items smaller than
    // min_item_evals evaluations
    const double target_items = std::max(
        1.0, std::min(tuning.items_per_slot * slots, static_cast<double>(total_work) / std::max(1, tuning.min_item_evals)));
    const double work_per_item = std::max(1.0, static_cast<double>(total_work) / target_items);
    // features per item of each node
    std::vector<int> per(M);
    long long plain_items = 0;
    for (int n = 0; n < M; n++) {
        const double w = static_cast<double>(node_counts[n]) * F;
        int parts = static_cast<int>(std::ceil(w / work_per_item));
        parts = std::max(1, std::min(parts, (F + g - 1) / g));
        per[n] = ((((F + parts - 1) / parts) + g - 1) / g) * g;
        plain_items += (F + per[n] - 1) / per[n];
    }
    // sample chunks where the level has too few items to fill the resident CTAs
    const long long want = static_cast<long long>(kChunkItemsPerSlot) * slots;
    const int k = chunk_features > 0 && plain_items < want ? static_cast<int>((want + plain_items - 1) / plain_items) : 1;
    // nodes of at least kChunkBigNodeSamples are cut into slices as well, however many items the level
    // has: their sweeps then share the frames of one slice in L2 instead of each CTA streaming a node
    // of frames from DRAM on its own (bounded by the groups' memory, max_groups)
    int groups = 0;
    items.clear();
    range.assign(M + 1, 0);
    std::vector<long long> work;
    for (int n = 0; n < M; n++) {
        range[n] = static_cast<int>(items.size());
        int chunks = std::min(k, node_counts[n] / kMinChunkSamples);
        if (chunk_features > 0 && node_counts[n] >= kChunkBigNodeSamples) chunks = std::max(chunks, 2);
        if (chunks > 1)   // slices of about kChunkTargetSamples, for the L2 locality of a chunk-major queue
            chunks = std::min(std::max(chunks, (node_counts[n] + kChunkTargetSamples - 1) / kChunkTargetSamples),
                              node_counts[n] / kMinChunkSamples);
        if (chunks > 1) {
            const int node_groups = (F + std::min(per[n], chunk_features) - 1) / std::min(per[n], chunk_features);
            if (groups + node_groups > max_groups) chunks = 1;   // over the group memory limit: whole-node items
        }
        const int pf = chunks > 1 ? std::min(per[n], chunk_features) : per[n];
        for (int f0 = 0; f0 < F; f0 += pf) {
            EvalItem it;
            it.node = n;
            it.f_begin = f0;
            it.f_end = std::min(F, f0 + pf);
            it.chunks = std::max(1, chunks);
            it.s_begin = 0;
            it.s_end = node_counts[n];
            it.group = -1;
            it.chunk = 0;
            if (chunks <= 1) {
                items.push_back(it);
                work.push_back(static_cast<long long>(node_counts[n]) * (it.f_end - it.f_begin));
                continue;
            }
            it.group = groups++;
            for (int c = 0; c < chunks; c++) {
                it.chunk = c;
                it.s_begin = static_cast<int>(static_cast<long long>(node_counts[n]) * c / chunks);
                it.s_end = static_cast<int>(static_cast<long long>(node_counts[n]) * (c + 1) / chunks);
                items.push_back(it);
                work.push_back(static_cast<long long>(it.s_end - it.s_begin) * (it.f_end - it.f_begin));
            }
        }
    }
    if (n_groups) *n_groups = groups;
    range[M] = static_cast<int>(items.size());
    const int n_items = static_cast<int>(items.size());
    order.resize(n_items);
    for (int i = 0; i < n_items; i++) order[i] = i;
    // chunked items first, chunk-major (by slice, then group: slice c of every node covers about the
    // same frames, since a node's samples are ordered by frame); then the rest, largest first
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const bool cx = items[x].chunks > 1, cy = items[y].chunks > 1;
        if (cx != cy) return cx;
        if (cx) return items[x].chunk != items[y].chunk ? items[x].chunk < items[y].chunk : items[x].group < items[y].group;
        return work[x] > work[y];
    });
}

void split_items_into_chunks(const std::vector<int>& node_counts, int chunk, int n_chunks,
                             std::vector<EvalItem>& items, std::vector<int>& range, std::vector<int>& order,
                             std::vector<int>& chunk_begin) {
    const int M = static_cast<int>(node_counts.size());
    std::vector<EvalItem> out;
    out.reserve(items.size() + static_cast<size_t>(M) * n_chunks);
    range.assign(M + 1, 0);
    int node = -1;
    for (const EvalItem& it : items) {   // items are node-major
        while (node < it.node) range[++node] = static_cast<int>(out.size());
        for (int f = it.f_begin; f < it.f_end;) {
            const int e = std::min(it.f_end, (f / chunk + 1) * chunk);
            EvalItem p = it;
            p.f_begin = f;
            p.f_end = e;
            out.push_back(p);
            f = e;
        }
    }
    while (node < M) range[++node] = static_cast<int>(out.size());
    items.swap(out);
    const int n = static_cast<int>(items.size());
    order.resize(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const int cx = items[x].f_begin / chunk, cy = items[y].f_begin / chunk;
        if (cx != cy) return cx < cy;
        return static_cast<long long>(node_counts[items[x].node]) * (items[x].f_end - items[x].f_begin) >
               static_cast<long long>(node_counts[items[y].node]) * (items[y].f_end - items[y].f_begin);
    });
    chunk_begin.assign(n_chunks + 1, n);
    for (int q = n - 1; q >= 0; q--) chunk_begin[items[order[q]].f_begin / chunk] = q;
    for (int c = n_chunks - 1; c >= 0; c--) chunk_begin[c] = std::min(chunk_begin[c], chunk_begin[c + 1]);
}

// Rows node by node, and their order sorted by (frame, Morton code), or with by_node by (node, frame,
// Morton code) for the sorted sample copy of the fused search.
void LevelEvaluator::stage_order(cf_context* ctx, const DsView& ds, const Sample* samples, const NodeDesc* nodes_dev,
                                 int M, const std::vector<int>& node_counts, long long rows, bool by_node) {
    h_row_base_.assign(M + 1, 0);
    for (int n = 0; n < M; n++) h_row_base_[n + 1] = h_row_base_[n] + node_counts[n];
    row_base_.reserve(M + 1);
    row_pos_.reserve(rows);
    row_label_.reserve(rows);
    pixel_key_.reserve(rows);
    pixel_key_sorted_.reserve(rows);
    row_ids_.reserve(rows);
    frame_order_.reserve(rows);
    CF_CUDA_CHECK(cudaMemcpyAsync(row_base_.get(), h_row_base_.data(), sizeof(long long) * (M + 1),
                                  cudaMemcpyHostToDevice, ctx->stream));
    flip_both_.reserve(1);
    CF_CUDA_CHECK(cudaMemsetAsync(flip_both_.get(), 0, sizeof(int), ctx->stream));
    int end_bit = 33;   // 32 bits of Morton code, then the frame, then (by_node) the node
    while (end_bit < 64 && (1ull << (end_bit - 32)) < static_cast<unsigned long long>(ds.n)) end_bit++;
    const int node_shift = by_node ? end_bit : 0;
    if (by_node)
        while (end_bit < 64 && (1ull << (end_bit - node_shift)) < static_cast<unsigned long long>(M)) end_bit++;
    launch(ctx, "stage_rows", dim3(static_cast<unsigned>((rows + 255) / 256)), dim3(256), 0, stage_rows_kernel,
           nodes_dev, row_base_.get(), M, rows, samples, node_shift, row_pos_.get(), row_label_.get(), pixel_key_.get(),
           row_ids_.get(),
           flip_both_.get());
    size_t temp = 0;
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, temp, pixel_key_.get(), pixel_key_sorted_.get(),
                                                  row_ids_.get(), frame_order_.get(), static_cast<int>(rows), 0,
                                                  end_bit, ctx->stream));
    sort_temp_.reserve(temp);
    CF_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(sort_temp_.get(), temp, pixel_key_.get(), pixel_key_sorted_.get(),
                                                  row_ids_.get(), frame_order_.get(), static_cast<int>(rows), 0,
                                                  end_bit, ctx->stream));
}

// ------------------------------------------------------------------------------------------------
void LevelEvaluator::evaluate(cf_context* ctx, const DsView& ds, const Sample* samples, const NodeDesc* nodes_dev,
                              const uint32_t* node_hist_dev, int M, const std::vector<int>& node_counts, int C,
                              const LevelFeatures& lf, cf_split* splits_dev, uint32_t* dump_left) {
    const int F = lf.F, T = lf.T;
    CF_REQUIRE(C >= 1 && C <= 256, "number of classes must be in [1, 256]");
    CF_REQUIRE(T >= 1 && T <= 4096, "number of thresholds must be in [1, 4096]");
    if (M == 0) return;
    tuning = EvalTuning::of(ctx);
    const int slots = ctx->num_sms * tuning.ctas_per_sm;
    const bool sharded = shard.world > 1;
    // staged bins: where the integral images do not fit in L2 (or on every level with stage_bins = 2);
    // the bins are bytes (T <= 255)
    long long rows = 0;
    for (int c : node_counts) rows += c;
    const size_t frame_bytes = static_cast<size_t>(ds.n) * ds.plane * (3 * sizeof(float) + sizeof(int2));
    const bool stage = tuning.stage_bins != 0 && !sharded && T <= 255 && rows > 0 && rows < INT_MAX &&
                       (tuning.stage_bins == 2 || frame_bytes > ctx->l2_bytes);
    // the staged search reads bytes instead of gathering, so it needs no L1: a larger histogram and
    // tiles of up to 32 features, and items of whole 32-feature rows (fewer, larger items: no CTAs
    // need to share a node's gathers)
    EvalTuning plan = tuning;
    if (stage) {
        plan.ft_max = kStagedFeatures;
        plan.bins_budget_words = std::max(plan.bins_budget_words, kStagedBinsWords);
        plan.feature_granule = kStageTile;
        plan.items_per_slot = std::min(plan.items_per_slot, kStagedItemsPerSlot);
        // (tiles kept at powers of two: the sample-group instance ran pass 2 in half the time of the
        // one-sample-per-thread instance with unrounded tiles, 51 against 108 ms on a level of 128 nodes)
    }
    int budget = 0;
    level_eval_smem(C, T, plan, &budget);
    // sample chunks of a node's items merge their counts on this device, so they are not sharded; a
    // chunked item covers at most the features of the smallest tile (all C classes present). Staged
    // levels chunk too: pass 2 of a level of one or two nodes has too few feature items to fill the
    // GPU otherwise (its tiles are powers of two, so a chunked item stays inside a 32-feature block)
    const int chunk_features =
        sharded ? 0 : tile_features(budget, C, T + 1, plan.ft_max, stage || plan.sample_groups != 0);
    int n_groups = 0;
    const int max_groups = static_cast<int>(kMaxChunkGroupBytes / (sizeof(uint32_t) * static_cast<size_t>(budget)));
    plan_level_items(node_counts, F, plan, slots, h_items_, h_range_, h_order_, chunk_features, &n_groups,
                     max_groups);
    int stage_chunk = 0, n_chunks = 0;
    size_t stage_bytes = 0;
    if (stage) {
        // feature chunks of whole 32-feature tiles whose table fits stage_max_mb, as even as possible
        const long long f_pad = (F + kStageTile - 1) / kStageTile * kStageTile;
        const long long max_bytes = static_cast<long long>(tuning.stage_max_mb) << 20;
        const long long tiles_max = std::max<long long>(1, max_bytes / rows / kStageTile);
        n_chunks = static_cast<int>((f_pad / kStageTile + tiles_max - 1) / tiles_max);
        stage_chunk = static_cast<int>((f_pad / kStageTile + n_chunks - 1) / n_chunks) * kStageTile;
        n_chunks = (F + stage_chunk - 1) / stage_chunk;
        stage_bytes = static_cast<size_t>(rows) * stage_chunk;
        split_items_into_chunks(node_counts, stage_chunk, n_chunks, h_items_, h_range_, h_order_, h_chunk_begin_);
    }
    last_stage_chunks = stage ? n_chunks : 0;
    const int n_items = static_cast<int>(h_items_.size());
    // this process's items: every position of the work order, or positions rank, rank + world, ...
    h_local_order_.clear();
    for (int q = sharded ? shard.rank : 0; q < n_items; q += sharded ? shard.world : 1)
        h_local_order_.push_back(h_order_[q]);
    const int n_local = static_cast<int>(h_local_order_.size());
    last_local_evals = 0;
    for (int id : h_local_order_)
        last_local_evals += static_cast<int64_t>(h_items_[id].s_end - h_items_[id].s_begin) *
                            (h_items_[id].f_end - h_items_[id].f_begin);
    items_.reserve(n_items);
    order_.reserve(n_items);
    item_range_.reserve(M + 1);
    cands_.reserve(n_items);
    queue_.reserve(1);
    CF_CUDA_CHECK(cudaMemcpyAsync(items_.get(), h_items_.data(), sizeof(EvalItem) * n_items, cudaMemcpyHostToDevice,
                                  ctx->stream));
    CF_CUDA_CHECK(cudaMemcpyAsync(order_.get(), h_local_order_.data(), sizeof(int) * std::max(1, n_local),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CF_CUDA_CHECK(cudaMemcpyAsync(item_range_.get(), h_range_.data(), sizeof(int) * (M + 1), cudaMemcpyHostToDevice,
                                  ctx->stream));
    CF_CUDA_CHECK(cudaMemsetAsync(queue_.get(), 0, sizeof(int), ctx->stream));
    if (n_groups > 0) {
        group_bins_.reserve(static_cast<size_t>(n_groups) * budget);
        group_count_.reserve(n_groups);
        CF_CUDA_CHECK(cudaMemsetAsync(group_bins_.get(), 0, sizeof(uint32_t) * n_groups * static_cast<size_t>(budget),
                                      ctx->stream));
        CF_CUDA_CHECK(cudaMemsetAsync(group_count_.get(), 0, sizeof(int) * n_groups, ctx->stream));
    }
    last_items = n_items;

    EvalArgs args;
    args.ds = ds;
    args.samples = samples;
    args.nodes = nodes_dev;
    args.node_hist = node_hist_dev;
    args.C = C;
    args.F = F;
    args.T = T;
    args.packs = lf.packs.get();
    args.sorted_thr = lf.sorted_thr.get();
    args.ranks = lf.ranks.get();
    args.items = items_.get();
    args.order = order_.get();
    args.n_items = n_local;
    args.queue = queue_.get();
    args.cands = cands_.get();
    args.ft_max = plan.ft_max;
    args.bins_budget = budget;
    args.group_bins = n_groups > 0 ? group_bins_.get() : nullptr;
    args.group_count = n_groups > 0 ? group_count_.get() : nullptr;
    args.dump_left = dump_left;
    node_consts_.reserve(sizeof(NodeConsts) * static_cast<size_t>(M));
    args.node_consts = reinterpret_cast<const NodeConsts*>(node_consts_.get());
    launch(ctx, "node_consts", dim3((M + 127) / 128), dim3(128), 0, node_consts_kernel, M, C, node_hist_dev,
           reinterpret_cast<NodeConsts*>(node_consts_.get()));
    if (stage) {
        queue_.reserve(n_chunks);
        CF_CUDA_CHECK(cudaMemsetAsync(queue_.get(), 0, sizeof(int) * n_chunks, ctx->stream));
        stage_order(ctx, ds, samples, nodes_dev, M, node_counts, rows, false);
        stage_.reserve(stage_bytes);
        args.staged = stage_.get();
        args.staged_rows = rows;
        args.row_label = row_label_.get();
        args.row_base = row_base_.get();
        args.staged_flip_both = flip_both_.get();
        StageArgs sa;
        sa.ds = ds;
        sa.samples = samples;
        sa.frame_order = frame_order_.get();
        sa.row_pos = row_pos_.get();
        sa.rows = rows;
        sa.packs = lf.packs.get();
        sa.sorted_thr = lf.sorted_thr.get();
        sa.T = T;
        sa.out = stage_.get();
        for (int c = 0; c < n_chunks; c++) {
            sa.f_first = c * stage_chunk;
            sa.n_feat = std::min(stage_chunk, F - sa.f_first);
            launch_stage_bins(ctx, sa);
            args.staged_f0 = sa.f_first;
            args.order = order_.get() + h_chunk_begin_[c];
            args.n_items = h_chunk_begin_[c + 1] - h_chunk_begin_[c];
            args.queue = queue_.get() + c;
            if (args.n_items > 0) launch_level_eval(ctx, args, std::min(args.n_items, slots), plan);
        }
    } else if (n_local > 0) {
        // one pass: where the frames exceed L2 (or sample_order = 2), a copy of the samples sorted by
        // (node, frame, Morton code) puts each CTA's samples in a compact patch of the frame; counts
        // do not depend on the order of a node's samples, and a slice of the sorted node still covers
        // a run of frames
        int key_bits = 32;
        while ((1ll << (key_bits - 32)) < ds.n) key_bits++;
        for (int m = M - 1; m > 0; m >>= 1) key_bits++;
        const bool sorted = tuning.sample_order != 0 && rows > 0 && rows < INT_MAX && key_bits <= 64 &&
                            (tuning.sample_order == 2 || frame_bytes > ctx->l2_bytes);
        if (sorted) {
            stage_order(ctx, ds, samples, nodes_dev, M, node_counts, rows, true);
            sorted_samples_.reserve(rows);
            launch(ctx, "gather_sorted_samples", dim3(static_cast<unsigned>((rows + 255) / 256)), dim3(256), 0,
                   gather_sorted_samples_kernel, rows, frame_order_.get(), row_pos_.get(), samples,
                   sorted_samples_.get());
            args.sorted_samples = sorted_samples_.get();
            args.row_base = row_base_.get();
        }
        launch_level_eval(ctx, args, std::min(n_local, slots), plan);
    }
    if (sharded) exchange(ctx, n_items);
    launch(ctx, "reduce_candidates", dim3((M + 7) / 8), dim3(256), 0, reduce_candidates_kernel, M, F,
           item_range_.get(), cands_.get(), lf.thr.get(), splits_dev);
}

// The candidate lists of this process's items go out in work-order position sequence (slot k holds
// position rank + k x world); the lists of every process come back and are placed by item, so the
// candidate array equals the one a single process computes.
void LevelEvaluator::exchange(cf_context* ctx, int n_items) {
    CF_REQUIRE(shard.allgather != nullptr, "sharded split search: no all-gather function");
    const int world = shard.world;
    const int per = (n_items + world - 1) / world;
    h_cands_.resize(n_items);
    CF_CUDA_CHECK(cudaMemcpyAsync(h_cands_.data(), cands_.get(), sizeof(ItemCandidates) * n_items,
                                  cudaMemcpyDeviceToHost, ctx->stream));
    CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    h_send_.assign(std::max(1, per), ItemCandidates{});
    for (int k = 0, q = shard.rank; q < n_items; k++, q += world) h_send_[k] = h_cands_[h_order_[q]];
    h_recv_.assign(static_cast<size_t>(std::max(1, per)) * world, ItemCandidates{});
    const size_t bytes = sizeof(ItemCandidates) * std::max(1, per);
    const int rc = shard.allgather(h_send_.data(), bytes, h_recv_.data(), shard.user);
    CF_REQUIRE(rc == 0, "sharded split search: the all-gather of candidate lists failed (" + std::to_string(rc) + ")");
    for (int r = 0; r < world; r++)
        for (int k = 0, q = r; q < n_items; k++, q += world) h_cands_[h_order_[q]] = h_recv_[static_cast<size_t>(r) * per + k];
    CF_CUDA_CHECK(cudaMemcpyAsync(cands_.get(), h_cands_.data(), sizeof(ItemCandidates) * n_items,
                                  cudaMemcpyHostToDevice, ctx->stream));
    CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
}

void plain_responses(cf_context* ctx, const DsView& ds, const Sample* samples_dev, long long start, int count,
                     const int8_t* feat_table, int F, double* resp1, double* resp2) {
    const unsigned fpb = std::min(F, 32);
    const unsigned spb = std::min(count, 4);
    dim3 grid((F + fpb - 1) / fpb, (count + spb - 1) / spb);
    launch(ctx, "plain_response", grid, dim3(spb, fpb), 0, plain_response_kernel, ds, samples_dev + start, count,
           feat_table, F, resp1, resp2);
}

void plain_scores(cf_context* ctx, int C, int F, int T, const uint32_t* counters, const uint32_t* node_hist,
                  double* scores) {
    const int tpb = std::min(F, 128);
    launch(ctx, "plain_score", dim3((F + tpb - 1) / tpb, T), dim3(tpb), 0, plain_score_kernel, counters, node_hist, C,
           F, T, scores);
}

void score_bounds(cf_context* ctx, int C, int F, int T, const uint32_t* counters, const uint32_t* node_hist,
                  float* lower, float* upper) {
    const int tpb = std::min(F, 128);
    launch(ctx, "score_bounds", dim3((F + tpb - 1) / tpb, T), dim3(tpb), 0, score_bounds_kernel, counters, node_hist,
           C, F, T, lower, upper);
}

void PlainNodeEvaluator::histograms(cf_context* ctx, const DsView& ds, const Sample* samples_dev, long long start,
                                    int count, int C, const int8_t* feat_table, const float* thr, int F, int T,
                                    int max_batch) {
    counters.reserve(static_cast<size_t>(F) * T * C * 2);
    CF_CUDA_CHECK(cudaMemsetAsync(counters.get(), 0, sizeof(uint32_t) * F * T * C * 2, ctx->stream));
    if (max_batch <= 0) max_batch = 50000;
    const int batch = std::min(count, max_batch);
    resp1.reserve(static_cast<size_t>(F) * batch);
    resp2.reserve(static_cast<size_t>(F) * batch);
    for (int b = 0; b < count; b += batch) {
        const int n = std::min(batch, count - b);
        plain_responses(ctx, ds, samples_dev, start + b, n, feat_table, F, resp1.get(), resp2.get());
        const int tpb = n <= 3000 ? 64 : 128;
        launch(ctx, "plain_histogram", dim3(T, F), dim3(tpb), sizeof(uint32_t) * 2 * C, plain_histogram_kernel,
               resp1.get(), resp2.get(), samples_dev + start + b, n, thr, F, T, C, counters.get());
    }
}

void host_window_argmax(const double* scores, int F, int T, int* best_f, int* best_t, double* best_s) {
    double m = -std::numeric_limits<double>::infinity();
    for (long long i = 0; i < static_cast<long long>(F) * T; i++) m = std::max(m, scores[i]);
    *best_f = 0;
    *best_t = 0;
    *best_s = m;
    for (int t = 0; t < T; t++)
        for (int f = 0; f < F; f++) {
            const double s = scores[static_cast<long long>(t) * F + f];
            if (m - s < 1e-13) {
                *best_f = f;
                *best_t = t;
                *best_s = s;
                return;
            }
        }
}

void PlainNodeEvaluator::evaluate_node(cf_context* ctx, const DsView& ds, const Sample* samples_dev, long long start,
                                       int count, const uint32_t* node_hist_dev, int C, const LevelFeatures& lf,
                                       int max_batch, cf_split* split_dev_out, cf_split* split_host_out) {
    const int F = lf.F, T = lf.T;
    histograms(ctx, ds, samples_dev, start, count, C, lf.feat.get(), lf.thr.get(), F, T, max_batch);
    scores.reserve(static_cast<size_t>(F) * T);
    plain_scores(ctx, C, F, T, counters.get(), node_hist_dev, scores.get());
    h_scores.resize(static_cast<size_t>(F) * T);
    CF_CUDA_CHECK(cudaMemcpyAsync(h_scores.data(), scores.get(), sizeof(double) * F * T, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    int bf, bt;
    double bs;
    host_window_argmax(h_scores.data(), F, T, &bf, &bt, &bs);
    float thr;
    CF_CUDA_CHECK(cudaMemcpy(&thr, lf.thr.get() + static_cast<long long>(bt) * F + bf, sizeof(float),
                             cudaMemcpyDeviceToHost));
    cf_split r;
    r.score = bs;
    r.feature = bf;
    r.threshold_index = bt;
    r.threshold = thr;
    r.flags = 0;
    if (split_host_out) *split_host_out = r;
    if (split_dev_out)
        CF_CUDA_CHECK(cudaMemcpyAsync(split_dev_out, &r, sizeof(cf_split), cudaMemcpyHostToDevice, ctx->stream));
    CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
}

}  // namespace cf

// ================================================================================================
// Allocation-free variant of the level-batched split search
// ================================================================================================
//
// Some callers cannot let a library allocate device memory: a host that owns all GPU memory
// through its own pool and hands out fixed buffers, or a latency-critical loop where cudaMalloc /
// cudaFree would synchronise the device and stall its other streams. For them this entry point
// takes every input and output as a device pointer and keeps its scratch (work items, candidate
// lists, node descriptors, prepared feature tables) in one fixed device array compiled into the
// library.
namespace cf {

__global__ void prepare_eval_features_kernel(int F, int T, const int8_t* __restrict__ feat,
                                             const float* __restrict__ thr, FeatParams* __restrict__ packs,
                                             float* __restrict__ sorted_thr, uint16_t* __restrict__ ranks);

namespace {

// 16 MiB per device, held by every GPU that loads the library until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr int kNoAllocMaxNodes = 65536;
constexpr int kNoAllocMaxItems = 65536;
constexpr long long kNoAllocMaxFeatureThresholds = 1LL << 20;  // features x thresholds
constexpr int kNoAllocMaxFeatures = 16384;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Status bits of the input check (noalloc_check_kernel).
constexpr int kBadImage = 1, kBadPixel = 2, kBadLabel = 4, kBadFlip = 8, kBadThreshold = 16;

// Checks the caller's device inputs before the split search reads them: every sample's image index,
// pixel, flip setting and label (the label must be counted in its node's histogram, because the
// kernel keeps histogram rows only for the classes a node's histogram holds), and every threshold
// (NaN would corrupt the sorted thresholds). Sets bits of *status; reads only checked indexes.
__global__ void noalloc_check_kernel(const Sample* __restrict__ samples, long long n,
                                     const NodeDesc* __restrict__ nodes, int M, const uint32_t* __restrict__ hist,
                                     int C, int num_images, int W, int H, const float* __restrict__ thr,
                                     long long n_thr, int* status) {
    int bad = 0;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n; i += stride) {
        const Sample s = samples[i];
        if (s.image >= static_cast<uint32_t>(num_images)) bad |= kBadImage;
        if (s.x >= W || s.y >= H) bad |= kBadPixel;
        if (s.flip > 2) bad |= kBadFlip;
        // the node owning sample i: the last node whose start is <= i (starts ascend, node 0 at 0)
        int lo = 0, hi = M - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (nodes[mid].start <= i) lo = mid;
            else hi = mid - 1;
        }
        if (s.label >= C || hist[static_cast<long long>(lo) * C + s.label] == 0u) bad |= kBadLabel;
    }
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n_thr; i += stride)
        if (isnan(thr[i])) bad |= kBadThreshold;
    if (bad) atomicOr(status, bad);
}

struct NoAllocLayout {
    size_t status, nodes, items, order, range, cands, queue, packs, sorted, ranks, total;
    NoAllocLayout(int M, int n_items, int F, int T) {
        auto a = [](size_t x) { return (x + 255) & ~size_t(255); };
        size_t o = 0;
        status = o;
        o += a(sizeof(int));
        nodes = o;
        o += a(sizeof(NodeDesc) * M);
        items = o;
        o += a(sizeof(EvalItem) * n_items);
        order = o;
        o += a(sizeof(int) * n_items);
        range = o;
        o += a(sizeof(int) * (M + 1));
        cands = o;
        o += a(sizeof(ItemCandidates) * n_items);
        queue = o;
        o += a(sizeof(int));
        packs = o;
        o += a(sizeof(FeatParams) * F);
        sorted = o;
        o += a(sizeof(float) * static_cast<size_t>(F) * T);
        ranks = o;
        o += a(sizeof(uint16_t) * static_cast<size_t>(F) * T);
        total = o;
    }
};

// Device address of the scratch array on the current device. In host code the array's name is a
// host-side stand-in, not a device address, so the address is looked up with the device current.
// The lookup is made on every call (it is cheap once the module is loaded), so no cached address
// outlives a device reset; the first call on a device loads the module, which is why that call
// should come before any stream capture.
char* noalloc_scratch() {
    void* p = nullptr;
    CF_CUDA_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    return static_cast<char*>(p);
}

}  // namespace
}  // namespace cf

extern "C" cf_status cf_evaluate_best_splits_noalloc(cf_context* ctx, const float* color, const int32_t* depth,
                                                     int num_images, int width, int height, int num_nodes,
                                                     const int64_t* node_offsets, const cf_sample* samples,
                                                     const uint32_t* node_histograms, int num_classes,
                                                     int num_features, int num_thresholds, const int8_t* features,
                                                     const float* thresholds, cf_split* best) {
    using namespace cf;
    return guard([&] {
        CF_REQUIRE(ctx && color && depth && node_offsets && samples && node_histograms && features && thresholds &&
                       best,
                   "cf_evaluate_best_splits_noalloc: NULL argument");
        CF_REQUIRE(num_images >= 1 && width >= 1 && height >= 1, "cf_evaluate_best_splits_noalloc: empty images");
        CF_REQUIRE(num_nodes >= 1 && num_nodes <= kNoAllocMaxNodes,
                   "cf_evaluate_best_splits_noalloc: num_nodes must be in [1, 65536]");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_evaluate_best_splits_noalloc: classes must be in [1, 256]");
        CF_REQUIRE(num_features >= 1 && num_features <= kNoAllocMaxFeatures && num_thresholds >= 1 &&
                       static_cast<long long>(num_features) * num_thresholds <= kNoAllocMaxFeatureThresholds,
                   "cf_evaluate_best_splits_noalloc: features x thresholds beyond the fixed scratch "
                   "(at most 16384 features and 2^20 feature-threshold pairs)");
        CF_REQUIRE(num_thresholds <= 4096, "cf_evaluate_best_splits_noalloc: thresholds must be in [1, 4096]");
        CF_REQUIRE(node_offsets[0] == 0, "cf_evaluate_best_splits_noalloc: node offsets must start at 0");
        make_current(ctx);
        const int M = num_nodes, F = num_features, T = num_thresholds, C = num_classes;
        // nodes and work items, sized as the level-batched evaluator sizes them
        std::vector<NodeDesc> nodes(M);
        std::vector<int> counts(M);
        for (int i = 0; i < M; i++) {
            const long long cnt = node_offsets[i + 1] - node_offsets[i];
            CF_REQUIRE(cnt >= 1 && cnt < (1LL << 31), "cf_evaluate_best_splits_noalloc: every node needs samples");
            nodes[i] = NodeDesc{node_offsets[i], static_cast<int>(cnt), i};
            counts[i] = static_cast<int>(cnt);
        }
        EvalTuning tuning = EvalTuning::of(ctx);
        const int slots = ctx->num_sms * tuning.ctas_per_sm;
        std::vector<EvalItem> items;
        std::vector<int> range, order;
        // fewer, larger items when the level would need more than the scratch holds
        for (;;) {
            plan_level_items(counts, F, tuning, slots, items, range, order);
            if (items.size() <= static_cast<size_t>(kNoAllocMaxItems) || tuning.items_per_slot < 0.01) break;
            tuning.items_per_slot *= 0.5;
        }
        CF_REQUIRE(items.size() <= static_cast<size_t>(kNoAllocMaxItems),
                   "cf_evaluate_best_splits_noalloc: level needs more than 65536 work items");
        const int n_items = static_cast<int>(items.size());

        const NoAllocLayout lay(M, n_items, F, T);
        CF_REQUIRE(lay.total <= kNoAllocScratchBytes, "cf_evaluate_best_splits_noalloc: level too large for the "
                                                      "16 MiB fixed scratch");
        char* base = noalloc_scratch();
        int* d_status = reinterpret_cast<int*>(base + lay.status);
        NodeDesc* d_nodes = reinterpret_cast<NodeDesc*>(base + lay.nodes);
        EvalItem* d_items = reinterpret_cast<EvalItem*>(base + lay.items);
        int* d_order = reinterpret_cast<int*>(base + lay.order);
        int* d_range = reinterpret_cast<int*>(base + lay.range);
        ItemCandidates* d_cands = reinterpret_cast<ItemCandidates*>(base + lay.cands);
        int* d_queue = reinterpret_cast<int*>(base + lay.queue);
        FeatParams* d_packs = reinterpret_cast<FeatParams*>(base + lay.packs);
        float* d_sorted = reinterpret_cast<float*>(base + lay.sorted);
        uint16_t* d_ranks = reinterpret_cast<uint16_t*>(base + lay.ranks);
        cudaStream_t st = ctx->stream;
        CF_CUDA_CHECK(cudaMemcpyAsync(d_nodes, nodes.data(), sizeof(NodeDesc) * M, cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(d_items, items.data(), sizeof(EvalItem) * n_items, cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(d_order, order.data(), sizeof(int) * n_items, cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(d_range, range.data(), sizeof(int) * (M + 1), cudaMemcpyHostToDevice, st));
        // the work queue counter and the check's status word are the scratch words that must start at
        // zero (the array keeps the previous call's contents)
        CF_CUDA_CHECK(cudaMemsetAsync(d_queue, 0, sizeof(int), st));
        CF_CUDA_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), st));
        // the caller's inputs are checked on the device before the split search indexes with them
        {
            const long long n = node_offsets[M];
            const long long n_thr = static_cast<long long>(F) * T;
            const long long work = std::max(n, n_thr);
            const int blocks = static_cast<int>(std::min<long long>((work + 255) / 256, 4LL * ctx->num_sms));
            launch(ctx, "noalloc_check", dim3(blocks), dim3(256), 0, noalloc_check_kernel,
                   reinterpret_cast<const Sample*>(samples), n, static_cast<const NodeDesc*>(d_nodes), M,
                   node_histograms, C, num_images, width, height, thresholds, n_thr, d_status);
            int status = 0;
            CF_CUDA_CHECK(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
            CF_CUDA_CHECK(cudaStreamSynchronize(st));
            std::string why;
            if (status & kBadImage) why += " image index >= num_images;";
            if (status & kBadPixel) why += " pixel outside the image;";
            if (status & kBadLabel) why += " label >= num_classes or not counted in its node's histogram;";
            if (status & kBadFlip) why += " flip setting > 2;";
            if (status & kBadThreshold) why += " NaN threshold;";
            CF_REQUIRE(status == 0, "cf_evaluate_best_splits_noalloc: invalid input:" + why);
        }
        launch(ctx, "prepare_features", dim3((F + 7) / 8), dim3(256), 0, prepare_eval_features_kernel, F, T, features,
               thresholds, d_packs, d_sorted, d_ranks);

        DsView ds;
        ds.color = color;
        ds.depth = reinterpret_cast<const int2*>(depth);
        ds.n = num_images;
        ds.width = width;
        ds.height = height;
        ds.plane = static_cast<long long>(width) * height;
        int budget = 0;
        level_eval_smem(C, T, tuning, &budget);
        EvalArgs args;
        args.ds = ds;
        args.samples = reinterpret_cast<const Sample*>(samples);
        args.nodes = d_nodes;
        args.node_hist = node_histograms;
        args.C = C;
        args.F = F;
        args.T = T;
        args.packs = d_packs;
        args.sorted_thr = d_sorted;
        args.ranks = d_ranks;
        args.items = d_items;
        args.order = d_order;
        args.n_items = n_items;
        args.queue = d_queue;
        args.cands = d_cands;
        args.ft_max = tuning.ft_max;
        args.bins_budget = budget;
        args.group_bins = nullptr;   // planned without sample chunks
        args.group_count = nullptr;
        args.dump_left = nullptr;
        launch_level_eval(ctx, args, std::min(n_items, slots), tuning);
        launch(ctx, "reduce_candidates", dim3((M + 7) / 8), dim3(256), 0, reduce_candidates_kernel, M, F, d_range,
               d_cands, thresholds, best);
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
    });
}
