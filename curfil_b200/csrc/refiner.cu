// The learned part: a per-pixel refinement network on top of the forest (project extension; the
// reference has no learned component on this path, its nearest hook is the disabled leaf-histogram
// refinement of random_forest_image.cpp:184-255).
//
// Input of pixel (x, y), D = 3C + 2 values: the forest's class probabilities p_c, their means over
// the (2 r1 + 1)^2 and (2 r2 + 1)^2 boxes around the pixel (clipped at the border), the pixel depth
// in metres / 5 (0 if invalid) and the depth-valid flag. Network: h = relu(W1 x + b1) (H hidden
// units), z = W2 h + b2 (C logits), softmax cross-entropy against the label. Training: Adam on
// minibatches of sampled labelled pixels; every gradient is a fixed-order sum (per-tile partial sums,
// then a sequential reduction), so training is deterministic.
//
// Parameters, float, contiguous: W1 [H][D], b1 [H], W2 [C][H], b2 [C].
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

#include "forest.h"

struct cf_refiner {
    cf_context* ctx = nullptr;
    int C = 0, D = 0, H = 0, P = 0;
    cf_refiner_config cfg{};
    cf::DevArray<float> params, m, v, grad;   // Adam state
    cf::DevArray<float> partial, loss_partial;
    int64_t step = 0;
    // scratch of feature planes and training data
    cf::DevArray<float> probs, mean1, mean2, tmp;
    cf::DevArray<float> X;
    cf::DevArray<int> Y, idx;
    cf::DevArray<cf::FrameDesc> frames;
};

namespace cf {

namespace {

constexpr int kTile = 64;        // samples per training tile
constexpr int kMaxHidden = 128;
constexpr int kMaxClasses = 64;

__device__ __forceinline__ float pixel_depth_m(const int2* D, int W, int x, int y) {
    const int2 c = __ldg(D + static_cast<long long>(y) * W + x);
    const int2 a = y > 0 ? __ldg(D + static_cast<long long>(y - 1) * W + x) : make_int2(0, 0);
    const int2 l = x > 0 ? __ldg(D + static_cast<long long>(y) * W + x - 1) : make_int2(0, 0);
    const int2 al = (x > 0 && y > 0) ? __ldg(D + static_cast<long long>(y - 1) * W + x - 1) : make_int2(0, 0);
    if (c.y - (l.y + a.y - al.y) != 1) return 0.0f;
    const int mm = static_cast<int>(static_cast<uint32_t>(c.x) -
                                    (static_cast<uint32_t>(l.x) + static_cast<uint32_t>(a.x) - static_cast<uint32_t>(al.x)));
    return mm > 0 ? static_cast<float>(mm) * 0.001f : 0.0f;
}

// box sums along x of every class plane: out[c][y][x] = sum_{|dx| <= r, clipped} in[c][y][x + dx]
__global__ void box_rows_kernel(const float* __restrict__ in, float* __restrict__ out, int planes, int W, int H, int r) {
    const long long n = static_cast<long long>(planes) * W * H;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % W);
        const long long row = i - x;
        const int x0 = max(0, x - r), x1 = min(W - 1, x + r);
        float s = 0.0f;
        for (int xx = x0; xx <= x1; xx++) s += in[row + xx];
        out[i] = s;
    }
}

// box means: column sums of the row sums divided by the clipped box area
__global__ void box_cols_kernel(const float* __restrict__ rows, float* __restrict__ out, int planes, int W, int H, int r) {
    const long long n = static_cast<long long>(planes) * W * H;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long plane_px = static_cast<long long>(W) * H;
        const long long c = i / plane_px;
        const long long p = i - c * plane_px;
        const int y = static_cast<int>(p / W), x = static_cast<int>(p - static_cast<long long>(y) * W);
        const int y0 = max(0, y - r), y1 = min(H - 1, y + r);
        const int x0 = max(0, x - r), x1 = min(W - 1, x + r);
        float s = 0.0f;
        for (int yy = y0; yy <= y1; yy++) s += rows[c * plane_px + static_cast<long long>(yy) * W + x];
        out[i] = s / static_cast<float>((y1 - y0 + 1) * (x1 - x0 + 1));
    }
}

struct FeaturePlanes {
    const float* p;       // [C][H][W]
    const float* m1;
    const float* m2;
    const int2* depth;    // integral image
    int W, H, C;
};

__device__ __forceinline__ float feature_at(const FeaturePlanes& f, int k, long long pix, int x, int y) {
    const long long plane = static_cast<long long>(f.W) * f.H;
    if (k < f.C) return f.p[k * plane + pix];
    if (k < 2 * f.C) return f.m1[(k - f.C) * plane + pix];
    if (k < 3 * f.C) return f.m2[(k - 2 * f.C) * plane + pix];
    const float d = pixel_depth_m(f.depth, f.W, x, y);
    return k == 3 * f.C ? d * 0.2f : (d > 0.0f ? 1.0f : 0.0f);
}

// X rows of listed pixels (x, y) of one frame
__global__ void gather_features_kernel(FeaturePlanes f, const int2* __restrict__ xy, int n, int D, float* __restrict__ X) {
    const long long total = static_cast<long long>(n) * D;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int r = static_cast<int>(i / D), k = static_cast<int>(i - static_cast<long long>(r) * D);
        const int2 q = xy[r];
        X[i] = feature_at(f, k, static_cast<long long>(q.y) * f.W + q.x, q.x, q.y);
    }
}

// Forward and backward of one tile of kTile samples (rows idx[s0 .. s0 + kTile) of X); writes the
// tile's gradient sums (scaled by 1/B) to partial[tile][P] and its loss sum to loss_partial[tile].
__global__ void __launch_bounds__(256)
mlp_tile_grad_kernel(const float* __restrict__ X, const int* __restrict__ Y, const int* __restrict__ idx, int B, int D,
                     int Hd, int C, const float* __restrict__ prm, float* __restrict__ partial,
                     float* __restrict__ loss_partial) {
    extern __shared__ __align__(16) float sm[];
    const int DP = D + 1;   // padded rows
    float* Xs = sm;                          // [kTile][DP]
    float* Hs = Xs + kTile * DP;             // [kTile][Hd]  activations
    float* Gs = Hs + kTile * Hd;             // [kTile][Hd]  d(pre-activation)
    float* Zs = Gs + kTile * Hd;             // [kTile][C]   logits, then d(logits)
    __shared__ float s_loss[kTile];
    const float* W1 = prm;
    const float* b1 = W1 + Hd * D;
    const float* W2 = b1 + Hd;
    const float* b2 = W2 + C * Hd;
    const int P = Hd * D + Hd + C * Hd + C;
    const int s0 = blockIdx.x * kTile;
    const int rows = min(kTile, B - s0);
    const float invB = 1.0f / static_cast<float>(B);
    for (int i = threadIdx.x; i < kTile * DP; i += blockDim.x) {
        const int r = i / DP, k = i - r * DP;
        Xs[i] = (r < rows && k < D) ? X[static_cast<long long>(idx[s0 + r]) * D + k] : 0.0f;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTile * Hd; i += blockDim.x) {
        const int r = i / Hd, j = i - r * Hd;
        float a = b1[j];
        const float* w = W1 + static_cast<long long>(j) * D;
        const float* x = Xs + r * DP;
        for (int k = 0; k < D; k++) a = fmaf(w[k], x[k], a);
        Hs[i] = r < rows ? fmaxf(a, 0.0f) : 0.0f;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTile * C; i += blockDim.x) {
        const int r = i / C, c = i - r * C;
        float z = b2[c];
        const float* w = W2 + static_cast<long long>(c) * Hd;
        const float* h = Hs + r * Hd;
        for (int j = 0; j < Hd; j++) z = fmaf(w[j], h[j], z);
        Zs[i] = z;
    }
    __syncthreads();
    // softmax cross-entropy per row; Zs becomes (softmax - onehot) / B
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < kTile; r += blockDim.x >> 5) {
        float* z = Zs + r * C;
        float m = -INFINITY;
        for (int c = lane; c < C; c += 32) m = fmaxf(m, z[c]);
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        float s = 0.0f;
        for (int c = lane; c < C; c += 32) s += expf(z[c] - m);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        const int y = r < rows ? Y[idx[s0 + r]] : -1;
        if (lane == 0) s_loss[r] = r < rows ? (logf(s) + m - z[y]) : 0.0f;
        __syncwarp();
        for (int c = lane; c < C; c += 32)
            z[c] = r < rows ? (expf(z[c] - m) / s - (c == y ? 1.0f : 0.0f)) * invB : 0.0f;
    }
    __syncthreads();
    // d(pre-activation) = (W2^T dz) * relu'
    for (int i = threadIdx.x; i < kTile * Hd; i += blockDim.x) {
        const int r = i / Hd, j = i - r * Hd;
        float g = 0.0f;
        for (int c = 0; c < C; c++) g = fmaf(W2[static_cast<long long>(c) * Hd + j], Zs[r * C + c], g);
        Gs[i] = Hs[i] > 0.0f ? g : 0.0f;
    }
    __syncthreads();
    float* out = partial + static_cast<long long>(blockIdx.x) * P;
    for (int i = threadIdx.x; i < Hd * D; i += blockDim.x) {     // dW1[j][k] = sum_r G[r][j] X[r][k]
        const int j = i / D, k = i - j * D;
        float a = 0.0f;
        for (int r = 0; r < kTile; r++) a = fmaf(Gs[r * Hd + j], Xs[r * DP + k], a);
        out[i] = a;
    }
    for (int j = threadIdx.x; j < Hd; j += blockDim.x) {          // db1
        float a = 0.0f;
        for (int r = 0; r < kTile; r++) a += Gs[r * Hd + j];
        out[Hd * D + j] = a;
    }
    for (int i = threadIdx.x; i < C * Hd; i += blockDim.x) {     // dW2[c][j] = sum_r dz[r][c] H[r][j]
        const int c = i / Hd, j = i - c * Hd;
        float a = 0.0f;
        for (int r = 0; r < kTile; r++) a = fmaf(Zs[r * C + c], Hs[r * Hd + j], a);
        out[Hd * D + Hd + i] = a;
    }
    for (int c = threadIdx.x; c < C; c += blockDim.x) {           // db2
        float a = 0.0f;
        for (int r = 0; r < kTile; r++) a += Zs[r * C + c];
        out[Hd * D + Hd + C * Hd + c] = a;
    }
    if (threadIdx.x == 0) {
        float l = 0.0f;
        for (int r = 0; r < kTile; r++) l += s_loss[r];
        loss_partial[blockIdx.x] = l;
    }
}

// grad = sum over tiles (fixed order); optionally one Adam step on the parameters
__global__ void mlp_reduce_adam_kernel(const float* __restrict__ partial, int tiles, int P, float* __restrict__ grad,
                                       float* __restrict__ prm, float* __restrict__ m, float* __restrict__ v,
                                       int adam, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    float g = 0.0f;
    for (int t = 0; t < tiles; t++) g += partial[static_cast<long long>(t) * P + i];
    grad[i] = g;
    if (!adam) return;
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    prm[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// per-pixel forward: probabilities (optional) and argmax label (lowest label on ties)
template <int kHd>
__global__ void __launch_bounds__(128)
mlp_predict_kernel(FeaturePlanes f, int D, int Hd, const float* __restrict__ prm, float* __restrict__ probs,
                   uint8_t* __restrict__ labels) {
    extern __shared__ __align__(16) float w[];
    const int C = f.C;
    const int P = Hd * D + Hd + C * Hd + C;
    for (int i = threadIdx.x; i < P; i += blockDim.x) w[i] = prm[i];
    __syncthreads();
    const float* W1 = w;
    const float* b1 = W1 + Hd * D;
    const float* W2 = b1 + Hd;
    const float* b2 = W2 + C * Hd;
    const long long plane = static_cast<long long>(f.W) * f.H;
    const long long pix = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (pix >= plane) return;
    const int y = static_cast<int>(pix / f.W), x = static_cast<int>(pix - static_cast<long long>(y) * f.W);
    float h[kHd];
#pragma unroll
    for (int j = 0; j < kHd; j++) h[j] = j < Hd ? b1[j] : 0.0f;
    for (int k = 0; k < D; k++) {
        const float xk = feature_at(f, k, pix, x, y);
#pragma unroll
        for (int j = 0; j < kHd; j++)
            if (j < Hd) h[j] = fmaf(W1[j * D + k], xk, h[j]);
    }
#pragma unroll
    for (int j = 0; j < kHd; j++) h[j] = fmaxf(h[j], 0.0f);
    auto logit = [&](int c) {
        float z = b2[c];
#pragma unroll
        for (int j = 0; j < kHd; j++)
            if (j < Hd) z = fmaf(W2[c * Hd + j], h[j], z);
        return z;
    };
    float mx = -INFINITY;
    int best = 0;
    for (int c = 0; c < C; c++) {
        const float z = logit(c);
        if (z > mx) {
            mx = z;
            best = c;
        }
    }
    if (labels) labels[pix] = static_cast<uint8_t>(best);
    if (probs) {
        float s = 0.0f;
        for (int c = 0; c < C; c++) s += expf(logit(c) - mx);
        for (int c = 0; c < C; c++) probs[c * plane + pix] = expf(logit(c) - mx) / s;
    }
}

// deterministic Glorot-uniform initialisation from a 64-bit mixer of (seed, index)
float init_value(uint32_t seed, int i, float a) {
    uint64_t z = (static_cast<uint64_t>(seed) << 32) ^ static_cast<uint64_t>(i) ^ 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = static_cast<double>(z >> 11) / 9007199254740992.0;   // [0, 1)
    return static_cast<float>((2.0 * u - 1.0) * a);
}

size_t tile_smem(int D, int Hd, int C) { return sizeof(float) * (kTile * (D + 1) + 2 * kTile * Hd + kTile * C); }

// forward/backward over B rows idx of X (device), gradient into r->grad; Adam step if `adam`
double run_batch(cf_refiner* r, const float* X, const int* Y, const int* idx, int B, bool adam) {
    cf_context* ctx = r->ctx;
    const int tiles = (B + kTile - 1) / kTile;
    r->partial.reserve(static_cast<size_t>(tiles) * r->P);
    r->loss_partial.reserve(tiles);
    const size_t smem = tile_smem(r->D, r->H, r->C);
    CF_CUDA_CHECK(cudaFuncSetAttribute(mlp_tile_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
    launch(ctx, "refiner_grad", dim3(tiles), dim3(256), smem, mlp_tile_grad_kernel, X, Y, idx, B, r->D, r->H, r->C,
           r->params.get(), r->partial.get(), r->loss_partial.get());
    float c1 = 1.0f, c2 = 1.0f;
    if (adam) {
        r->step++;
        c1 = 1.0f - std::pow(0.9f, static_cast<float>(r->step));
        c2 = 1.0f - std::pow(0.999f, static_cast<float>(r->step));
    }
    launch(ctx, "refiner_adam", dim3((r->P + 255) / 256), dim3(256), 0, mlp_reduce_adam_kernel, r->partial.get(),
           tiles, r->P, r->grad.get(), r->params.get(), r->m.get(), r->v.get(), adam ? 1 : 0, r->cfg.learning_rate,
           0.9f, 0.999f, 1e-8f, c1, c2);
    std::vector<float> lp(tiles);
    CF_CUDA_CHECK(cudaMemcpyAsync(lp.data(), r->loss_partial.get(), sizeof(float) * tiles, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    double loss = 0;
    for (float x : lp) loss += x;
    return loss / B;
}

// forest probabilities and their box means of dataset frames [first, first + count) into the scratch
// planes (frames one at a time), calling `per_frame(i, planes)` for each
template <typename F>
void for_each_frame_features(cf_refiner* r, cf_forest* forest, cf_dataset* ds, int first, int count, F per_frame) {
    cf_context* ctx = r->ctx;
    const int C = r->C, W = ds->width, H = ds->height;
    const long long plane = static_cast<long long>(W) * H;
    r->probs.reserve(plane * C);
    r->mean1.reserve(plane * C);
    r->mean2.reserve(plane * C);
    r->tmp.reserve(plane * C);
    r->frames.reserve(1);
    const int grid = ctx->num_sms * 8;
    for (int i = 0; i < count; i++) {
        FrameDesc fr;
        fr.color = ds->color.get() + (first + i) * plane * 3;
        fr.depth = ds->depth.get() + (first + i) * plane;
        fr.probs = r->probs.get();
        fr.labels = nullptr;
        fr.width = W;
        fr.height = H;
        fr.first_block = 0;
        fr.pad = 0;
        CF_CUDA_CHECK(cudaMemcpyAsync(r->frames.get(), &fr, sizeof(fr), cudaMemcpyHostToDevice, ctx->stream));
        classify_frames(ctx, forest, r->frames.get(), 1, classify_blocks_for(W, H));
        launch(ctx, "refiner_box", dim3(grid), dim3(256), 0, box_rows_kernel, r->probs.get(), r->tmp.get(), C, W, H,
               r->cfg.radius1);
        launch(ctx, "refiner_box", dim3(grid), dim3(256), 0, box_cols_kernel, r->tmp.get(), r->mean1.get(), C, W, H,
               r->cfg.radius1);
        launch(ctx, "refiner_box", dim3(grid), dim3(256), 0, box_rows_kernel, r->probs.get(), r->tmp.get(), C, W, H,
               r->cfg.radius2);
        launch(ctx, "refiner_box", dim3(grid), dim3(256), 0, box_cols_kernel, r->tmp.get(), r->mean2.get(), C, W, H,
               r->cfg.radius2);
        FeaturePlanes f{r->probs.get(), r->mean1.get(), r->mean2.get(), fr.depth, W, H, C};
        per_frame(i, f);
    }
}

}  // namespace

}  // namespace cf

using namespace cf;

extern "C" {

cf_status cf_refiner_create(cf_context* ctx, int num_classes, const cf_refiner_config* config, cf_refiner** out) {
    return guard([&] {
        CF_REQUIRE(ctx && config && out, "cf_refiner_create: NULL argument");
        CF_REQUIRE(num_classes >= 2 && num_classes <= kMaxClasses, "cf_refiner_create: classes must be in [2, 64]");
        CF_REQUIRE(config->hidden >= 1 && config->hidden <= kMaxHidden, "cf_refiner_create: hidden must be in [1, 128]");
        CF_REQUIRE(config->radius1 >= 0 && config->radius2 >= 0, "cf_refiner_create: radii must be >= 0");
        CF_REQUIRE(config->epochs >= 0 && config->batch >= 1 && config->pixels_per_image >= 1,
                   "cf_refiner_create: epochs >= 0, batch >= 1, pixels_per_image >= 1");
        CF_REQUIRE(config->learning_rate > 0.0f, "cf_refiner_create: learning rate must be > 0");
        make_current(ctx);
        auto* r = new cf_refiner();
        std::unique_ptr<cf_refiner> own(r);
        r->ctx = ctx;
        r->cfg = *config;
        r->C = num_classes;
        r->D = 3 * num_classes + 2;
        r->H = config->hidden;
        r->P = r->H * r->D + r->H + r->C * r->H + r->C;
        CF_REQUIRE(tile_smem(r->D, r->H, r->C) + 1024 <= ctx->smem_per_block_optin,
                   "cf_refiner_create: network too wide for one training tile in shared memory");
        std::vector<float> init(r->P, 0.0f);
        const float a1 = std::sqrt(6.0f / static_cast<float>(r->D + r->H));
        const float a2 = std::sqrt(6.0f / static_cast<float>(r->H + r->C));
        for (int i = 0; i < r->H * r->D; i++) init[i] = init_value(config->seed, i, a1);
        for (int i = 0; i < r->C * r->H; i++) init[r->H * r->D + r->H + i] = init_value(config->seed, r->P + i, a2);
        r->params.reserve(r->P);
        r->m.reserve(r->P);
        r->v.reserve(r->P);
        r->grad.reserve(r->P);
        CF_CUDA_CHECK(cudaMemcpyAsync(r->params.get(), init.data(), sizeof(float) * r->P, cudaMemcpyHostToDevice,
                                      ctx->stream));
        CF_CUDA_CHECK(cudaMemsetAsync(r->m.get(), 0, sizeof(float) * r->P, ctx->stream));
        CF_CUDA_CHECK(cudaMemsetAsync(r->v.get(), 0, sizeof(float) * r->P, ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
        context_retain(ctx);
        *out = own.release();
    });
}

cf_status cf_refiner_destroy(cf_refiner* r) {
    return guard([&] {
        if (!r) return;
        cf_context* ctx = r->ctx;
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        delete r;
        context_release(ctx);
    });
}

cf_status cf_refiner_params(cf_refiner* r, float* get, const float* set, int* num_params) {
    return guard([&] {
        CF_REQUIRE(r, "cf_refiner_params: refiner is NULL");
        make_current(r->ctx);
        if (num_params) *num_params = r->P;
        if (set) {
            CF_CUDA_CHECK(cudaMemcpyAsync(r->params.get(), set, sizeof(float) * r->P, cudaMemcpyHostToDevice,
                                          r->ctx->stream));
            CF_CUDA_CHECK(cudaMemsetAsync(r->m.get(), 0, sizeof(float) * r->P, r->ctx->stream));
            CF_CUDA_CHECK(cudaMemsetAsync(r->v.get(), 0, sizeof(float) * r->P, r->ctx->stream));
            r->step = 0;
        }
        if (get)
            CF_CUDA_CHECK(cudaMemcpyAsync(get, r->params.get(), sizeof(float) * r->P, cudaMemcpyDeviceToHost,
                                          r->ctx->stream));
        CF_CUDA_CHECK(cudaStreamSynchronize(r->ctx->stream));
    });
}

cf_status cf_refiner_loss_grad(cf_refiner* r, int n, const float* features, const uint8_t* labels, float* grad,
                               double* loss) {
    return guard([&] {
        CF_REQUIRE(r && features && labels && grad && loss, "cf_refiner_loss_grad: NULL argument");
        CF_REQUIRE(n >= 1, "cf_refiner_loss_grad: no samples");
        for (int i = 0; i < n; i++) CF_REQUIRE(labels[i] < r->C, "cf_refiner_loss_grad: label >= number of classes");
        make_current(r->ctx);
        cudaStream_t st = r->ctx->stream;
        DevArray<float> X;
        DevArray<int> Y, idx;
        X.reserve(static_cast<size_t>(n) * r->D);
        Y.reserve(n);
        idx.reserve(n);
        std::vector<int> y(labels, labels + n), id(n);
        for (int i = 0; i < n; i++) id[i] = i;
        CF_CUDA_CHECK(cudaMemcpyAsync(X.get(), features, sizeof(float) * n * r->D, cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(Y.get(), y.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(idx.get(), id.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
        *loss = run_batch(r, X.get(), Y.get(), idx.get(), n, false);
        CF_CUDA_CHECK(cudaMemcpyAsync(grad, r->grad.get(), sizeof(float) * r->P, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
    });
}

cf_status cf_refiner_features(cf_refiner* r, cf_forest* forest, cf_dataset* ds, int frame, int n, const int32_t* xy,
                              float* out) {
    return guard([&] {
        CF_REQUIRE(r && forest && ds && xy && out, "cf_refiner_features: NULL argument");
        CF_REQUIRE(forest->C == r->C && ds->ctx == r->ctx && forest->ctx == r->ctx, "cf_refiner_features: mismatch");
        CF_REQUIRE(frame >= 0 && frame < ds->n && n >= 1, "cf_refiner_features: frame or count");
        for (int i = 0; i < n; i++)
            CF_REQUIRE(xy[2 * i] >= 0 && xy[2 * i] < ds->width && xy[2 * i + 1] >= 0 && xy[2 * i + 1] < ds->height,
                       "cf_refiner_features: pixel outside the frame");
        make_current(r->ctx);
        cudaStream_t st = r->ctx->stream;
        DevArray<int2> d_xy;
        DevArray<float> X;
        d_xy.reserve(n);
        X.reserve(static_cast<size_t>(n) * r->D);
        CF_CUDA_CHECK(cudaMemcpyAsync(d_xy.get(), xy, sizeof(int2) * n, cudaMemcpyHostToDevice, st));
        for_each_frame_features(r, forest, ds, frame, 1, [&](int, const FeaturePlanes& f) {
            launch(r->ctx, "refiner_gather", dim3(r->ctx->num_sms * 4), dim3(256), 0, gather_features_kernel, f,
                   d_xy.get(), n, r->D, X.get());
        });
        CF_CUDA_CHECK(cudaMemcpyAsync(out, X.get(), sizeof(float) * n * r->D, cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
    });
}

cf_status cf_refiner_train(cf_refiner* r, cf_forest* forest, cf_dataset* ds, int first, int count,
                           const uint8_t* labels, const uint8_t* ignored, float* loss_per_epoch) {
    return guard([&] {
        CF_REQUIRE(r && forest && ds && labels, "cf_refiner_train: NULL argument");
        CF_REQUIRE(forest->C == r->C && ds->ctx == r->ctx && forest->ctx == r->ctx, "cf_refiner_train: mismatch");
        CF_REQUIRE(first >= 0 && count >= 1 && first + count <= ds->n, "cf_refiner_train: image range");
        make_current(r->ctx);
        cudaStream_t st = r->ctx->stream;
        const int W = ds->width, H = ds->height, C = r->C, D = r->D;
        const long long plane = static_cast<long long>(W) * H;
        // training pixels: pixels_per_image per frame, uniform over the labelled (not ignored) pixels
        std::mt19937 gen(r->cfg.seed ^ 0x51ED2701u);
        std::vector<std::vector<int2>> xy(count);
        std::vector<int> ys;
        for (int i = 0; i < count; i++) {
            std::vector<int> ok;
            for (long long p = 0; p < plane; p++) {
                const uint8_t l = labels[i * plane + p];
                CF_REQUIRE(l < C, "cf_refiner_train: label >= number of classes");
                if (!(ignored && ignored[l])) ok.push_back(static_cast<int>(p));
            }
            CF_REQUIRE(!ok.empty(), "cf_refiner_train: a frame has no labelled pixel");
            std::uniform_int_distribution<size_t> pick(0, ok.size() - 1);
            for (int s = 0; s < r->cfg.pixels_per_image; s++) {
                const int p = ok[pick(gen)];
                xy[i].push_back(make_int2(p % W, p / W));
                ys.push_back(labels[i * plane + p]);
            }
        }
        const int N = static_cast<int>(ys.size());
        r->X.reserve(static_cast<size_t>(N) * D);
        r->Y.reserve(N);
        r->idx.reserve(N);
        CF_CUDA_CHECK(cudaMemcpyAsync(r->Y.get(), ys.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
        DevArray<int2> d_xy;
        d_xy.reserve(r->cfg.pixels_per_image);
        for_each_frame_features(r, forest, ds, first, count, [&](int i, const FeaturePlanes& f) {
            CF_CUDA_CHECK(cudaMemcpyAsync(d_xy.get(), xy[i].data(), sizeof(int2) * xy[i].size(), cudaMemcpyHostToDevice,
                                          st));
            launch(r->ctx, "refiner_gather", dim3(r->ctx->num_sms * 4), dim3(256), 0, gather_features_kernel, f,
                   d_xy.get(), static_cast<int>(xy[i].size()), D,
                   r->X.get() + static_cast<size_t>(i) * r->cfg.pixels_per_image * D);
            CF_CUDA_CHECK(cudaStreamSynchronize(st));   // d_xy is reused by the next frame
        });
        std::vector<int> order(N);
        for (int i = 0; i < N; i++) order[i] = i;
        const int B = std::min(N, r->cfg.batch);
        for (int e = 0; e < r->cfg.epochs; e++) {
            std::shuffle(order.begin(), order.end(), gen);
            CF_CUDA_CHECK(cudaMemcpyAsync(r->idx.get(), order.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
            double sum = 0;
            int batches = 0;
            for (int b = 0; b + B <= N; b += B) {
                sum += run_batch(r, r->X.get(), r->Y.get(), r->idx.get() + b, B, true);
                batches++;
            }
            if (loss_per_epoch) loss_per_epoch[e] = static_cast<float>(sum / std::max(1, batches));
        }
    });
}

cf_status cf_refiner_predict(cf_refiner* r, cf_forest* forest, cf_dataset* ds, int first, int count,
                             float* probabilities, uint8_t* labels) {
    return guard([&] {
        CF_REQUIRE(r && forest && ds, "cf_refiner_predict: NULL argument");
        CF_REQUIRE(forest->C == r->C && ds->ctx == r->ctx && forest->ctx == r->ctx, "cf_refiner_predict: mismatch");
        CF_REQUIRE(first >= 0 && count >= 1 && first + count <= ds->n, "cf_refiner_predict: image range");
        make_current(r->ctx);
        const long long plane = static_cast<long long>(ds->width) * ds->height;
        const size_t smem = sizeof(float) * r->P;
        auto kernel = r->H <= 32 ? mlp_predict_kernel<32> : r->H <= 64 ? mlp_predict_kernel<64> : mlp_predict_kernel<128>;
        CF_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        for_each_frame_features(r, forest, ds, first, count, [&](int i, const FeaturePlanes& f) {
            launch(r->ctx, "refiner_predict", dim3(static_cast<unsigned>((plane + 127) / 128)), dim3(128), smem,
                   kernel, f, r->D, r->H, r->params.get(),
                   probabilities ? probabilities + static_cast<long long>(i) * r->C * plane : nullptr,
                   labels ? labels + static_cast<long long>(i) * plane : nullptr);
        });
        CF_CUDA_CHECK(cudaStreamSynchronize(r->ctx->stream));
    });
}

}  // extern "C"
