// Routing of a level's samples on the GPU.
//
// Follows RandomTreeTrain::train (random_tree.h:1296-1406): every sample of a node goes left when
// its double response is <= the split threshold (NaN goes right). With horizontal flipping Both,
// a sample whose flipped response disagrees is split into a NoFlip copy on its own side and a
// Flip copy on the other side. Children keep the parent's sample order (a stable partition via
// two exclusive scans), children ids follow the parent order (left, right), and only children
// that are impure and hold at least minSampleCount samples continue into the next level.
#include <algorithm>

#include "route.h"

namespace cf {

void DevTree::reserve(int cap, int C_) {
    capacity = cap;
    C = C_;
    level.reserve(cap);
    left.reserve(cap);
    feature_id.reserve(cap);
    feature.reserve(static_cast<size_t>(cap) * 11);
    threshold.reserve(cap);
    score.reserve(cap);
    hist.reserve(static_cast<size_t>(cap) * C);
    nsamp.reserve(cap);
}

void RouteBuffers::reserve(long long n, int M, int C) {
    cntL.reserve(n + 1);
    cntR.reserve(n + 1);
    posL.reserve(n + 1);
    posR.reserve(n + 1);
    code.reserve(n + 1);
    child_hist.reserve(static_cast<size_t>(2) * M * C);
    cont.reserve(2 * static_cast<size_t>(M) + 1);
    cont_count.reserve(2 * static_cast<size_t>(M) + 1);
    next_idx.reserve(2 * static_cast<size_t>(M) + 1);
    next_off.reserve(2 * static_cast<size_t>(M) + 1);
    err.reserve(1);
}

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t warp_prefix = warp > 0 ? s_warp[warp - 1] : 0;
    *total = s_warp[kScanThreads / 32 - 1];
    return warp_prefix + x - v;
}

// Exclusive scan of one tile of kScanTile elements (index n reads as 0); block total to `sums`.
__global__ void __launch_bounds__(kScanThreads)
scan_tiles_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, long long n_plus, long long n_in,
                  uint32_t* __restrict__ sums) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const long long base = static_cast<long long>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const long long i = base + k;
        v[k] = (i < n_in) ? in[i] : 0u;
        local += v[k];
    }
    uint32_t total;
    uint32_t prefix = block_exclusive_scan(local, s_warp, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const long long i = base + k;
        if (i < n_plus) out[i] = prefix;
        prefix += v[k];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
scan_add_kernel(uint32_t* __restrict__ out, long long n_plus, const uint32_t* __restrict__ offsets) {
    const long long base = static_cast<long long>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
    const uint32_t add = offsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const long long i = base + k;
        if (i < n_plus) out[i] += add;
    }
}

// Side(s) of every sample under its node's split; child histograms (weight 2 for Both).
// code: 0 left, 1 right, 2 left NoFlip + right Flip, 3 left Flip + right NoFlip.
__global__ void __launch_bounds__(256)
route_flags_kernel(DsView ds, const Sample* __restrict__ samples, const int* __restrict__ sample_node, long long n,
                   const cf_split* __restrict__ splits, const FeatParams* __restrict__ packs, int C,
                   uint32_t* __restrict__ cntL, uint32_t* __restrict__ cntR, uint8_t* __restrict__ code,
                   uint32_t* __restrict__ child_hist) {
    const long long s = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    int keyL = -1, keyR = -1;
    uint32_t wL = 0, wR = 0;
    if (s < n) {
        const int node = sample_node[s];
        const cf_split sp = splits[node];
        const FeatParams fp = packs[sp.feature];
        const Sample smp = samples[s];
        const double thr = static_cast<double>(sp.threshold);
        uint8_t c;
        if (smp.flip == 2) {
            const bool a = sample_response(ds, smp, fp, false) <= thr;
            const bool b = sample_response(ds, smp, fp, true) <= thr;
            if (a == b) {
                c = a ? 0 : 1;
                if (a) wL = 2; else wR = 2;
            } else {
                c = a ? 2 : 3;
                wL = 1;
                wR = 1;
            }
        } else {
            const bool a = sample_response(ds, smp, fp, smp.flip == 1) <= thr;
            c = a ? 0 : 1;
            if (a) wL = 1; else wR = 1;
        }
        code[s] = c;
        cntL[s] = wL > 0 ? 1u : 0u;
        cntR[s] = wR > 0 ? 1u : 0u;
        if (wL) keyL = (node * 2 + 0) * C + smp.label;
        if (wR) keyR = (node * 2 + 1) * C + smp.label;
    }
    // warp-aggregated histogram increments
    {
        const unsigned peers = __match_any_sync(kFull, keyL);
        const uint32_t sum = __reduce_add_sync(peers, wL);
        if (keyL >= 0 && static_cast<int>(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(child_hist + keyL, sum);
    }
    {
        const unsigned peers = __match_any_sync(kFull, keyR);
        const uint32_t sum = __reduce_add_sync(peers, wR);
        if (keyR >= 0 && static_cast<int>(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(child_hist + keyR, sum);
    }
}

struct ChildrenArgs {
    const NodeDesc* nodes;
    int M;
    const uint32_t* posL;
    const uint32_t* posR;
    const cf_split* splits;
    const int8_t* feat;   // sorted [11][F]
    int F;
    const uint32_t* child_hist;
    int C;
    int level;
    int min_samples;
    int next_tree_base;
    int32_t* t_level;
    int32_t* t_left;
    int32_t* t_feature_id;
    int8_t* t_feature;
    float* t_threshold;
    double* t_score;
    uint32_t* t_hist;
    uint32_t* t_nsamp;
    uint32_t* cont;
    uint32_t* cont_count;
    int* err;
};

__global__ void __launch_bounds__(128)
children_kernel(ChildrenArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.M) return;
    const NodeDesc nd = a.nodes[i];
    const long long b = nd.start, e = nd.start + nd.count;
    const uint32_t nl = a.posL[e] - a.posL[b];
    const uint32_t nr = a.posR[e] - a.posR[b];
    if (nl == 0 || nr == 0) atomicOr(a.err, 1);
    const cf_split sp = a.splits[i];
    const int pi = nd.tree_index;
    const int cl = a.next_tree_base + 2 * i;
    a.t_left[pi] = cl;
    for (int r = 0; r < 11; r++) a.t_feature[static_cast<long long>(pi) * 11 + r] = a.feat[r * a.F + sp.feature];
    a.t_threshold[pi] = sp.threshold;
    a.t_score[pi] = sp.score;
    a.t_feature_id[pi] = sp.feature;
    for (int side = 0; side < 2; side++) {
        const int ci = cl + side;
        const uint32_t cnt = side == 0 ? nl : nr;
        const uint32_t* h = a.child_hist + (static_cast<long long>(i) * 2 + side) * a.C;
        a.t_level[ci] = a.level + 1;
        a.t_left[ci] = -1;
        for (int r = 0; r < 11; r++) a.t_feature[static_cast<long long>(ci) * 11 + r] = 0;
        a.t_threshold[ci] = __int_as_float(0x7fc00000);
        a.t_score[ci] = __longlong_as_double(0x7ff8000000000000ULL);
        a.t_feature_id[ci] = -1;
        a.t_nsamp[ci] = cnt;
        int nonzero = 0;
        for (int c = 0; c < a.C; c++) {
            const uint32_t v = h[c];
            a.t_hist[static_cast<long long>(ci) * a.C + c] = v;
            nonzero += v != 0;
        }
        // shouldContinueGrowing (random_tree.h:1182-1191)
        const bool cont = nonzero > 1 && cnt >= static_cast<uint32_t>(a.min_samples);
        a.cont[2 * i + side] = cont ? 1u : 0u;
        a.cont_count[2 * i + side] = cont ? cnt : 0u;
    }
}

__global__ void __launch_bounds__(256)
scatter_kernel(long long n, const Sample* __restrict__ samples, const int* __restrict__ sample_node,
               const uint8_t* __restrict__ code, const uint32_t* __restrict__ posL, const uint32_t* __restrict__ posR,
               const NodeDesc* __restrict__ nodes, const uint32_t* __restrict__ cont,
               const uint32_t* __restrict__ next_idx, const uint32_t* __restrict__ next_off,
               Sample* __restrict__ samples_out, int* __restrict__ node_out) {
    const long long s = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int node = sample_node[s];
    const long long start = nodes[node].start;
    const uint8_t c = code[s];
    Sample smp = samples[s];
    const bool toL = c != 1;
    const bool toR = c != 0;
    if (toL && cont[2 * node]) {
        Sample o = smp;
        if (c == 2) o.flip = 0;
        if (c == 3) o.flip = 1;
        const long long d = next_off[2 * node] + (posL[s] - posL[start]);
        samples_out[d] = o;
        node_out[d] = static_cast<int>(next_idx[2 * node]);
    }
    if (toR && cont[2 * node + 1]) {
        Sample o = smp;
        if (c == 2) o.flip = 1;
        if (c == 3) o.flip = 0;
        const long long d = next_off[2 * node + 1] + (posR[s] - posR[start]);
        samples_out[d] = o;
        node_out[d] = static_cast<int>(next_idx[2 * node + 1]);
    }
}

__global__ void __launch_bounds__(128)
next_nodes_kernel(int M2, int C, int next_tree_base, const uint32_t* __restrict__ cont,
                  const uint32_t* __restrict__ cont_count, const uint32_t* __restrict__ next_idx,
                  const uint32_t* __restrict__ next_off, const uint32_t* __restrict__ child_hist,
                  NodeDesc* __restrict__ next_nodes, uint32_t* __restrict__ next_hist) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M2 || !cont[c]) return;
    const int j = static_cast<int>(next_idx[c]);
    NodeDesc d;
    d.start = next_off[c];
    d.count = static_cast<int>(cont_count[c]);
    d.tree_index = next_tree_base + c;
    next_nodes[j] = d;
    for (int k = 0; k < C; k++) next_hist[static_cast<long long>(j) * C + k] = child_hist[static_cast<long long>(c) * C + k];
}

}  // namespace

void Scanner::exclusive(cf_context* ctx, const uint32_t* in, uint32_t* out, long long n) {
    scan_level(ctx, in, out, n, n + 1, 0);
}

// Scans n_out elements (index >= n_in reads as 0) of `in` into `out`; tile sums are scanned
// recursively and added back.
void Scanner::scan_level(cf_context* ctx, const uint32_t* in, uint32_t* out, long long n_in, long long n_out,
                         size_t depth) {
    const long long tiles = (n_out + kScanTile - 1) / kScanTile;
    CF_REQUIRE(depth < kMaxDepth, "scan: input too large");
    DevArray<uint32_t>& sums = temps_[2 * depth];
    DevArray<uint32_t>& offsets = temps_[2 * depth + 1];
    sums.reserve(tiles + 1);
    offsets.reserve(tiles + 1);
    launch(ctx, "scan", dim3(static_cast<unsigned>(tiles)), dim3(kScanThreads), 0, scan_tiles_kernel, in, out, n_out,
           n_in, sums.get());
    if (tiles == 1) return;
    scan_level(ctx, sums.get(), offsets.get(), tiles, tiles, depth + 1);
    launch(ctx, "scan_add", dim3(static_cast<unsigned>(tiles)), dim3(kScanThreads), 0, scan_add_kernel, out, n_out,
           offsets.get());
}

RouteResult route_level(cf_context* ctx, const DsView& ds, const Sample* samples, const int* sample_node, long long n,
                        const NodeDesc* nodes, int M, const cf_split* splits, const LevelFeatures& lf, int C,
                        int level, int min_samples, int next_tree_base, bool scatter, DevTree& tree,
                        RouteBuffers& rb, Scanner& scan, Sample* samples_out, int* node_out, NodeDesc* next_nodes,
                        uint32_t* next_hist) {
    rb.reserve(n, M, C);
    CF_CUDA_CHECK(cudaMemsetAsync(rb.child_hist.get(), 0, sizeof(uint32_t) * 2 * M * C, ctx->stream));
    CF_CUDA_CHECK(cudaMemsetAsync(rb.err.get(), 0, sizeof(int), ctx->stream));
    launch(ctx, "route_flags", dim3(static_cast<unsigned>((n + 255) / 256)), dim3(256), 0, route_flags_kernel, ds,
           samples, sample_node, n, splits, lf.packs.get(), C, rb.cntL.get(), rb.cntR.get(), rb.code.get(),
           rb.child_hist.get());
    scan.exclusive(ctx, rb.cntL.get(), rb.posL.get(), n);
    scan.exclusive(ctx, rb.cntR.get(), rb.posR.get(), n);
    ChildrenArgs ca;
    ca.nodes = nodes;
    ca.M = M;
    ca.posL = rb.posL.get();
    ca.posR = rb.posR.get();
    ca.splits = splits;
    ca.feat = lf.feat.get();
    ca.F = lf.F;
    ca.child_hist = rb.child_hist.get();
    ca.C = C;
    ca.level = level;
    ca.min_samples = min_samples;
    ca.next_tree_base = next_tree_base;
    ca.t_level = tree.level.get();
    ca.t_left = tree.left.get();
    ca.t_feature_id = tree.feature_id.get();
    ca.t_feature = tree.feature.get();
    ca.t_threshold = tree.threshold.get();
    ca.t_score = tree.score.get();
    ca.t_hist = tree.hist.get();
    ca.t_nsamp = tree.nsamp.get();
    ca.cont = rb.cont.get();
    ca.cont_count = rb.cont_count.get();
    ca.err = rb.err.get();
    launch(ctx, "route_children", dim3((M + 127) / 128), dim3(128), 0, children_kernel, ca);
    RouteResult res;
    CF_CUDA_CHECK(cudaMemcpyAsync(&res.empty_child, rb.err.get(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (scatter) {
        scan.exclusive(ctx, rb.cont.get(), rb.next_idx.get(), 2LL * M);
        scan.exclusive(ctx, rb.cont_count.get(), rb.next_off.get(), 2LL * M);
        launch(ctx, "route_scatter", dim3(static_cast<unsigned>((n + 255) / 256)), dim3(256), 0, scatter_kernel, n,
               samples, sample_node, rb.code.get(), rb.posL.get(), rb.posR.get(), nodes, rb.cont.get(),
               rb.next_idx.get(), rb.next_off.get(), samples_out, node_out);
        launch(ctx, "route_next_nodes", dim3((2 * M + 127) / 128), dim3(128), 0, next_nodes_kernel, 2 * M, C,
               next_tree_base, rb.cont.get(), rb.cont_count.get(), rb.next_idx.get(), rb.next_off.get(),
               rb.child_hist.get(), next_nodes, next_hist);
        uint32_t totals[2];
        CF_CUDA_CHECK(cudaMemcpyAsync(&totals[0], rb.next_idx.get() + 2LL * M, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                      ctx->stream));
        CF_CUDA_CHECK(cudaMemcpyAsync(&totals[1], rb.next_off.get() + 2LL * M, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                      ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
        res.next_nodes = static_cast<int>(totals[0]);
        res.next_samples = totals[1];
    } else {
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    }
    return res;
}

}  // namespace cf
