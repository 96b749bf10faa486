// Integral images on the GPU (kernel a) and the device-resident dataset.
//
// The reference integrates each channel sequentially in double with a Kahan carry and stores
// float (colour) / int (depth) (image.cpp:236-277, 531-556). For integer-valued input the
// double scan is exact, so an exact 32-bit integer scan followed by one round-to-nearest
// conversion (__uint2float_rn) gives bit-identical colour integrals. Depth sums are kept as
// wrapping 32-bit integers: box differences stay exact even where the reference's int
// integral overflows (1280x960 frames at up to 5 m).
//
// Two passes: a warp-per-row inclusive scan of the five channels, then a thread-per-column
// running sum down the rows. Traffic: 5 B/px read raw, 20 B/px written, then 20 B/px read and
// written again.
#include <algorithm>
#include <cstring>

#include "features.h"

namespace cf {

namespace {

constexpr int kRowWarps = 8;

__global__ void __launch_bounds__(kRowWarps * 32)
integral_rows_kernel(const uint8_t* __restrict__ rgb, const uint16_t* __restrict__ depth, int count, int W, int H,
                     uint32_t* __restrict__ color_out, int2* __restrict__ depth_out) {
    const int lane = threadIdx.x & 31;
    const long long row = static_cast<long long>(blockIdx.x) * kRowWarps + (threadIdx.x >> 5);
    if (row >= static_cast<long long>(count) * H) return;
    const long long img = row / H;
    const int y = static_cast<int>(row - img * H);
    const long long plane = static_cast<long long>(W) * H;
    const uint8_t* src_rgb = rgb + (img * plane + static_cast<long long>(y) * W) * 3;
    const uint16_t* src_d = depth + img * plane + static_cast<long long>(y) * W;
    uint32_t* dst_c = color_out + img * 3 * plane + static_cast<long long>(y) * W;
    int2* dst_d = depth_out + img * plane + static_cast<long long>(y) * W;
    uint32_t carry[5] = {0, 0, 0, 0, 0};
    for (int x0 = 0; x0 < W; x0 += 32) {
        const int x = x0 + lane;
        uint32_t v[5] = {0, 0, 0, 0, 0};
        if (x < W) {
            v[0] = src_rgb[x * 3 + 0];
            v[1] = src_rgb[x * 3 + 1];
            v[2] = src_rgb[x * 3 + 2];
            v[3] = src_d[x];
            v[4] = v[3] > 0 ? 1u : 0u;
        }
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
            for (int c = 0; c < 5; c++) {
                const uint32_t o = __shfl_up_sync(0xffffffffu, v[c], off);
                if (lane >= off) v[c] += o;
            }
        }
#pragma unroll
        for (int c = 0; c < 5; c++) v[c] += carry[c];
        if (x < W) {
            dst_c[x] = v[0];
            dst_c[plane + x] = v[1];
            dst_c[2 * plane + x] = v[2];
            dst_d[x] = make_int2(static_cast<int>(v[3]), static_cast<int>(v[4]));
        }
#pragma unroll
        for (int c = 0; c < 5; c++) carry[c] = __shfl_sync(0xffffffffu, v[c], 31);
    }
}

__global__ void __launch_bounds__(256)
integral_cols_kernel(int count, int W, int H, uint32_t* __restrict__ color, int2* __restrict__ depth) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const long long img = blockIdx.y;
    if (x >= W || img >= count) return;
    const long long plane = static_cast<long long>(W) * H;
    uint32_t* c0 = color + img * 3 * plane + x;
    int2* d0 = depth + img * plane + x;
    uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0;
    int y = 0;
    for (; y + 4 <= H; y += 4) {
        uint32_t r0[4], r1[4], r2[4];
        int2 rd[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const long long o = static_cast<long long>(y + k) * W;
            r0[k] = c0[o];
            r1[k] = c0[plane + o];
            r2[k] = c0[2 * plane + o];
            rd[k] = d0[o];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const long long o = static_cast<long long>(y + k) * W;
            a0 += r0[k];
            a1 += r1[k];
            a2 += r2[k];
            a3 += static_cast<uint32_t>(rd[k].x);
            a4 += static_cast<uint32_t>(rd[k].y);
            reinterpret_cast<float*>(c0)[o] = __uint2float_rn(a0);
            reinterpret_cast<float*>(c0)[plane + o] = __uint2float_rn(a1);
            reinterpret_cast<float*>(c0)[2 * plane + o] = __uint2float_rn(a2);
            d0[o] = make_int2(static_cast<int>(a3), static_cast<int>(a4));
        }
    }
    for (; y < H; y++) {
        const long long o = static_cast<long long>(y) * W;
        a0 += c0[o];
        a1 += c0[plane + o];
        a2 += c0[2 * plane + o];
        const int2 rd = d0[o];
        a3 += static_cast<uint32_t>(rd.x);
        a4 += static_cast<uint32_t>(rd.y);
        reinterpret_cast<float*>(c0)[o] = __uint2float_rn(a0);
        reinterpret_cast<float*>(c0)[plane + o] = __uint2float_rn(a1);
        reinterpret_cast<float*>(c0)[2 * plane + o] = __uint2float_rn(a2);
        d0[o] = make_int2(static_cast<int>(a3), static_cast<int>(a4));
    }
}

// RGBDImage::resizeImage (image.cpp:450-475) applied to integral images: the w x h integrals go to the
// top-left corner of the W x H frames, colour NaN and depth {0, 0} everywhere else.
__global__ void pad_integral_kernel(const float* __restrict__ color_in, const int2* __restrict__ depth_in, int count,
                                    int w, int h, int W, int H, float* __restrict__ color_out,
                                    int2* __restrict__ depth_out) {
    const long long plane = static_cast<long long>(W) * H, small = static_cast<long long>(w) * h;
    const long long total = plane * count;
    const float nan = __int_as_float(0x7fc00000);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long img = i / plane;
        const long long p = i - img * plane;
        const int y = static_cast<int>(p / W), x = static_cast<int>(p - static_cast<long long>(y) * W);
        float* c = color_out + img * 3 * plane + p;
        if (x < w && y < h) {
            const long long q = img * small + static_cast<long long>(y) * w + x;
            const float* s = color_in + img * 3 * small + static_cast<long long>(y) * w + x;
            c[0] = s[0];
            c[plane] = s[small];
            c[2 * plane] = s[2 * small];
            depth_out[i] = depth_in[q];
        } else {
            c[0] = nan;
            c[plane] = nan;
            c[2 * plane] = nan;
            depth_out[i] = make_int2(0, 0);
        }
    }
}

}  // namespace

// Integrates `count` raw frames (device pointers) into the given integral buffers.
void integrate_frames(cf_context* ctx, const uint8_t* rgb_dev, uint16_t* depth_dev, int count, int W, int H,
                      float* color_out, int2* depth_out, cudaStream_t stream, int preprocess) {
    if (stream == nullptr) stream = ctx->stream;
    if (preprocess & kPreFillDepth) fill_depth_frames(ctx, depth_dev, count, W, H, stream);
    const long long rows = static_cast<long long>(count) * H;
    launch_on(ctx, stream, "integral_rows", dim3(static_cast<unsigned>((rows + kRowWarps - 1) / kRowWarps)),
           dim3(kRowWarps * 32), 0, integral_rows_kernel, rgb_dev, depth_dev, count, W, H,
           reinterpret_cast<uint32_t*>(color_out), depth_out);
    launch_on(ctx, stream, "integral_cols", dim3((W + 255) / 256, count), dim3(256), 0, integral_cols_kernel, count, W, H,
           reinterpret_cast<uint32_t*>(color_out), depth_out);
    if (preprocess & kPreCieLab) lab_color_integral(ctx, rgb_dev, count, W, H, color_out, stream);
}

DsView view_of(const cf_dataset* ds) {
    DsView v;
    v.color = ds->color.get();
    v.depth = ds->depth.get();
    v.n = ds->n;
    v.width = ds->width;
    v.height = ds->height;
    v.plane = static_cast<long long>(ds->width) * ds->height;
    return v;
}

}  // namespace cf

extern "C" {

cf_status cf_dataset_create(cf_context* ctx, int num_images, int width, int height, cf_dataset** out) {
    return cf::guard([&] {
        CF_REQUIRE(ctx && out, "cf_dataset_create: NULL argument");
        CF_REQUIRE(num_images > 0 && width > 0 && height > 0, "cf_dataset_create: empty dataset");
        CF_REQUIRE(width <= 65535 && height <= 65535, "cf_dataset_create: frames wider or higher than 65535 px");
        cf::make_current(ctx);
        auto* ds = new cf_dataset();
        ds->ctx = ctx;
        ds->n = num_images;
        ds->width = width;
        ds->height = height;
        const size_t plane = static_cast<size_t>(width) * height;
        try {
            ds->color.reserve(plane * 3 * num_images);
            ds->depth.reserve(plane * num_images);
        } catch (...) {
            delete ds;
            throw;
        }
        cf::context_retain(ctx);
        *out = ds;
    });
}

cf_status cf_dataset_destroy(cf_dataset* ds) {
    return cf::guard([&] {
        if (!ds) return;
        cf_context* ctx = ds->ctx;
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        {
            // the dataset's training buffers stay with the context for the next dataset
            std::lock_guard<std::mutex> lock(ctx->mu);
            if (ds->trainer && ctx->spare_trainer == nullptr) {
                ctx->spare_trainer = ds->trainer;
                ctx->spare_trainer_free = ds->trainer_free;
                ds->trainer = nullptr;
            }
        }
        delete ds;
        cf::context_release(ctx);
    });
}

cf_status cf_dataset_info(cf_dataset* ds, int* num_images, int* width, int* height) {
    return cf::guard([&] {
        CF_REQUIRE(ds, "cf_dataset_info: ds is NULL");
        if (num_images) *num_images = ds->n;
        if (width) *width = ds->width;
        if (height) *height = ds->height;
    });
}

cf_status cf_dataset_upload_raw(cf_dataset* ds, int first, int count, const uint8_t* rgb, const uint16_t* depth_mm,
                                int device_pointers) {
    return cf_dataset_upload_raw_ex(ds, first, count, rgb, depth_mm, device_pointers, 0, 0);
}

cf_status cf_dataset_upload_raw_ex(cf_dataset* ds, int first, int count, const uint8_t* rgb, const uint16_t* depth_mm,
                                   int device_pointers, int fill_depth, int cie_lab) {
    return cf::guard([&] {
        CF_REQUIRE(ds && rgb && depth_mm, "cf_dataset_upload_raw: NULL argument");
        CF_REQUIRE(first >= 0 && count >= 0 && first + count <= ds->n, "cf_dataset_upload_raw: image range");
        if (count == 0) return;
        cf_context* ctx = ds->ctx;
        cf::make_current(ctx);
        const size_t plane = static_cast<size_t>(ds->width) * ds->height;
        const int pre = (fill_depth ? cf::kPreFillDepth : 0) | (cie_lab ? cf::kPreCieLab : 0);
        if (!device_pointers || fill_depth) {
            // bounded staging (the depth frames are filled in place there); chunks keep the extra
            // memory small for large datasets
            const cudaMemcpyKind kind = device_pointers ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
            const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(count, (256u << 20) / (plane * 5))));
            ds->raw_rgb.reserve(plane * 3 * chunk);
            ds->raw_depth.reserve(plane * chunk);
            for (int i = 0; i < count; i += chunk) {
                const int c = std::min(chunk, count - i);
                CF_CUDA_CHECK(cudaMemcpyAsync(ds->raw_rgb.get(), rgb + plane * 3 * i, plane * 3 * c, kind, ctx->stream));
                CF_CUDA_CHECK(cudaMemcpyAsync(ds->raw_depth.get(), depth_mm + plane * i, plane * 2 * c, kind, ctx->stream));
                cf::integrate_frames(ctx, ds->raw_rgb.get(), ds->raw_depth.get(), c, ds->width, ds->height,
                                     ds->color.get() + plane * 3 * (first + i), ds->depth.get() + plane * (first + i),
                                     ctx->stream, pre);
            }
            CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
        } else {
            // without depth filling the frames are only read
            cf::integrate_frames(ctx, rgb, const_cast<uint16_t*>(depth_mm), count, ds->width, ds->height,
                                 ds->color.get() + plane * 3 * first, ds->depth.get() + plane * first, ctx->stream,
                                 pre);
        }
    });
}

cf_status cf_dataset_upload_raw_padded(cf_dataset* ds, int first, int count, int width, int height, const uint8_t* rgb,
                                       const uint16_t* depth_mm, int device_pointers, int fill_depth, int cie_lab) {
    return cf::guard([&] {
        CF_REQUIRE(ds && rgb && depth_mm, "cf_dataset_upload_raw_padded: NULL argument");
        CF_REQUIRE(first >= 0 && count >= 0 && first + count <= ds->n, "cf_dataset_upload_raw_padded: image range");
        CF_REQUIRE(width >= 1 && height >= 1 && width <= ds->width && height <= ds->height,
                   "cf_dataset_upload_raw_padded: frames must be at most as large as the dataset's");
        if (count == 0) return;
        cf_context* ctx = ds->ctx;
        cf::make_current(ctx);
        const size_t small = static_cast<size_t>(width) * height;
        const size_t plane = static_cast<size_t>(ds->width) * ds->height;
        const int pre = (fill_depth ? cf::kPreFillDepth : 0) | (cie_lab ? cf::kPreCieLab : 0);
        const cudaMemcpyKind kind = device_pointers ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(count, (256u << 20) / (small * 25))));
        cf::DevArray<uint8_t> raw_rgb;
        cf::DevArray<uint16_t> raw_depth;
        cf::DevArray<float> color;
        cf::DevArray<int2> depth;
        raw_rgb.reserve(small * 3 * chunk);
        raw_depth.reserve(small * chunk);
        color.reserve(small * 3 * chunk);
        depth.reserve(small * chunk);
        for (int i = 0; i < count; i += chunk) {
            const int c = std::min(chunk, count - i);
            CF_CUDA_CHECK(cudaMemcpyAsync(raw_rgb.get(), rgb + small * 3 * i, small * 3 * c, kind, ctx->stream));
            CF_CUDA_CHECK(cudaMemcpyAsync(raw_depth.get(), depth_mm + small * i, small * 2 * c, kind, ctx->stream));
            cf::integrate_frames(ctx, raw_rgb.get(), raw_depth.get(), c, width, height, color.get(), depth.get(),
                                 ctx->stream, pre);
            const long long total = static_cast<long long>(plane) * c;
            const int grid = static_cast<int>(std::min<long long>(ctx->num_sms * 8LL, (total + 255) / 256));
            cf::launch(ctx, "pad_integral", dim3(grid), dim3(256), 0, cf::pad_integral_kernel, color.get(), depth.get(),
                       c, width, height, ds->width, ds->height, ds->color.get() + plane * 3 * (first + i),
                       ds->depth.get() + plane * (first + i));
        }
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_dataset_upload_integral(cf_dataset* ds, int first, int count, const float* color, const int32_t* depth) {
    return cf::guard([&] {
        CF_REQUIRE(ds && color && depth, "cf_dataset_upload_integral: NULL argument");
        CF_REQUIRE(first >= 0 && count >= 0 && first + count <= ds->n, "cf_dataset_upload_integral: image range");
        cf_context* ctx = ds->ctx;
        cf::make_current(ctx);
        const size_t plane = static_cast<size_t>(ds->width) * ds->height;
        CF_CUDA_CHECK(cudaMemcpyAsync(ds->color.get() + plane * 3 * first, color, plane * 3 * count * sizeof(float),
                                      cudaMemcpyHostToDevice, ctx->stream));
        std::vector<int2> inter(plane);
        for (int i = 0; i < count; i++) {
            const int32_t* src = depth + plane * 2 * i;
            for (size_t p = 0; p < plane; p++) inter[p] = make_int2(src[p], src[plane + p]);
            CF_CUDA_CHECK(cudaMemcpyAsync(ds->depth.get() + plane * (first + i), inter.data(), plane * sizeof(int2),
                                          cudaMemcpyHostToDevice, ctx->stream));
            CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
        }
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_dataset_download_integral(cf_dataset* ds, int first, int count, float* color, int32_t* depth) {
    return cf::guard([&] {
        CF_REQUIRE(ds, "cf_dataset_download_integral: ds is NULL");
        CF_REQUIRE(first >= 0 && count >= 0 && first + count <= ds->n, "cf_dataset_download_integral: image range");
        cf_context* ctx = ds->ctx;
        cf::make_current(ctx);
        const size_t plane = static_cast<size_t>(ds->width) * ds->height;
        if (color)
            CF_CUDA_CHECK(cudaMemcpyAsync(color, ds->color.get() + plane * 3 * first, plane * 3 * count * sizeof(float),
                                          cudaMemcpyDeviceToHost, ctx->stream));
        if (depth) {
            std::vector<int2> inter(plane);
            for (int i = 0; i < count; i++) {
                CF_CUDA_CHECK(cudaMemcpyAsync(inter.data(), ds->depth.get() + plane * (first + i), plane * sizeof(int2),
                                              cudaMemcpyDeviceToHost, ctx->stream));
                CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
                int32_t* dst = depth + plane * 2 * i;
                for (size_t p = 0; p < plane; p++) {
                    dst[p] = inter[p].x;
                    dst[plane + p] = inter[p].y;
                }
            }
        }
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

}  // extern "C"
