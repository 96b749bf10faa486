// Image preprocessing on the device (RGBDImage, image.cpp:89-105, 279-377):
//   - depth filling: RGBDImage::fillDepth runs four passes over the depth image, each replacing a
//     missing (0) depth by its already-processed neighbour: from the right (x = W-2 .. 0 takes x+1),
//     from the left (x = 1 .. W-1 takes x-1), from the top (y = 1 .. H-1 takes y-1), from the bottom
//     (y = H-2 .. 0 takes y+1). Rows (and columns) are independent, so one thread runs one row (or
//     column) of a pass; the result is bit-identical.
//   - CIELab: the reference converts with Vigra's RGB2LabFunctor<double> (linear RGB in [0, 255]), a
//     library not available here, so the published CIE 1976 L*a*b* definition is restated: RGB / 255
//     -> XYZ with the ITU-R BT.709 primaries (D65), then L* = 116 f(Y/Yn) - 16, a* = 500 (f(X/Xn) -
//     f(Y/Yn)), b* = 200 (f(Y/Yn) - f(Z/Zn)), f(t) = cbrt(t) for t > (6/29)^3 else t / (3 (6/29)^2) +
//     4/29, white (Xn, Yn, Zn) = (0.950456, 1, 1.088754). Values are rounded to float as the reference
//     stores them (setColor), then integrated in double and rounded to float (the reference's Kahan
//     scan in double, image.cpp:250-277, to within the final float rounding).
#include "features.h"

namespace cf {

namespace {

__global__ void fill_depth_rows_kernel(uint16_t* __restrict__ d, long long rows, int W) {
    const long long row = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (row >= rows) return;
    uint16_t* r = d + row * W;
    for (int x = W - 2; x >= 0; x--)
        if (!r[x]) r[x] = r[x + 1];
    for (int x = 1; x < W; x++)
        if (!r[x]) r[x] = r[x - 1];
}

__global__ void fill_depth_cols_kernel(uint16_t* __restrict__ d, int count, int W, int H) {
    const long long col = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (col >= static_cast<long long>(count) * W) return;
    const long long img = col / W;
    const int x = static_cast<int>(col - img * W);
    uint16_t* c = d + img * W * static_cast<long long>(H) + x;
    for (int y = 1; y < H; y++)
        if (!c[static_cast<long long>(y) * W]) c[static_cast<long long>(y) * W] = c[static_cast<long long>(y - 1) * W];
    for (int y = H - 2; y >= 0; y--)
        if (!c[static_cast<long long>(y) * W]) c[static_cast<long long>(y) * W] = c[static_cast<long long>(y + 1) * W];
}

__device__ __forceinline__ double lab_f(double t) {
    const double e = 216.0 / 24389.0;   // (6/29)^3
    return t > e ? cbrt(t) : t * (841.0 / 108.0) + 4.0 / 29.0;
}

// RGB (uint8, interleaved) -> L*a*b* float planes [n][3][H][W]
__global__ void rgb_to_lab_kernel(const uint8_t* __restrict__ rgb, long long pixels, long long plane,
                                  float* __restrict__ lab) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= pixels) return;
    const double r = rgb[3 * i] / 255.0, g = rgb[3 * i + 1] / 255.0, b = rgb[3 * i + 2] / 255.0;
    const double X = 0.412453 * r + 0.357580 * g + 0.180423 * b;
    const double Y = 0.212671 * r + 0.715160 * g + 0.072169 * b;
    const double Z = 0.019334 * r + 0.119193 * g + 0.950227 * b;
    const double fx = lab_f(X / 0.950456), fy = lab_f(Y), fz = lab_f(Z / 1.088754);
    const long long img = i / plane, p = i - img * plane;
    float* out = lab + img * 3 * plane + p;
    out[0] = static_cast<float>(116.0 * fy - 16.0);
    out[plane] = static_cast<float>(500.0 * (fx - fy));
    out[2 * plane] = static_cast<float>(200.0 * (fy - fz));
}

// row prefix sums in double of float planes (one thread per row of a plane)
__global__ void prefix_rows_double_kernel(const float* __restrict__ in, double* __restrict__ out, long long rows, int W) {
    const long long row = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (row >= rows) return;
    double s = 0.0;
    for (int x = 0; x < W; x++) {
        s += static_cast<double>(in[row * W + x]);
        out[row * W + x] = s;
    }
}

// column prefix sums of the row sums (one thread per column of a plane), rounded to float
__global__ void prefix_cols_float_kernel(const double* __restrict__ in, float* __restrict__ out, long long planes,
                                         int W, int H) {
    const long long col = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (col >= planes * W) return;
    const long long pl = col / W;
    const int x = static_cast<int>(col - pl * W);
    const long long base = pl * W * static_cast<long long>(H) + x;
    double s = 0.0;
    for (int y = 0; y < H; y++) {
        s += in[base + static_cast<long long>(y) * W];
        out[base + static_cast<long long>(y) * W] = static_cast<float>(s);
    }
}

// 2-D inclusive prefix sums of int32 planes with 32-bit wrap-around (box differences stay exact):
// rows first (one thread per row), then columns (one thread per column), in place
__global__ void prefix_rows_int_kernel(int32_t* __restrict__ d, long long rows, int W) {
    const long long row = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (row >= rows) return;
    uint32_t* r = reinterpret_cast<uint32_t*>(d) + row * W;
    uint32_t s = 0;
    for (int x = 0; x < W; x++) {
        s += r[x];
        r[x] = s;
    }
}

__global__ void prefix_cols_int_kernel(int32_t* __restrict__ d, long long planes, int W, int H) {
    const long long col = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (col >= planes * W) return;
    const long long pl = col / W;
    const int x = static_cast<int>(col - pl * W);
    uint32_t* c = reinterpret_cast<uint32_t*>(d) + pl * W * static_cast<long long>(H) + x;
    uint32_t s = 0;
    for (int y = 0; y < H; y++) {
        s += c[static_cast<long long>(y) * W];
        c[static_cast<long long>(y) * W] = s;
    }
}

}  // namespace

void fill_depth_frames(cf_context* ctx, uint16_t* depth, int count, int W, int H, cudaStream_t stream) {
    if (stream == nullptr) stream = ctx->stream;
    const long long rows = static_cast<long long>(count) * H;
    launch_on(ctx, stream, "fill_depth", dim3(static_cast<unsigned>((rows + 127) / 128)), dim3(128), 0,
              fill_depth_rows_kernel, depth, rows, W);
    const long long cols = static_cast<long long>(count) * W;
    launch_on(ctx, stream, "fill_depth", dim3(static_cast<unsigned>((cols + 127) / 128)), dim3(128), 0,
              fill_depth_cols_kernel, depth, count, W, H);
}

void rgb_to_lab(cf_context* ctx, const uint8_t* rgb, int count, int W, int H, float* lab, cudaStream_t stream) {
    if (stream == nullptr) stream = ctx->stream;
    const long long plane = static_cast<long long>(W) * H;
    const long long px = plane * count;
    launch_on(ctx, stream, "rgb_to_lab", dim3(static_cast<unsigned>((px + 255) / 256)), dim3(256), 0,
              rgb_to_lab_kernel, rgb, px, plane, lab);
}

void lab_color_integral(cf_context* ctx, const uint8_t* rgb, int count, int W, int H, float* color_out,
                        cudaStream_t stream) {
    if (stream == nullptr) stream = ctx->stream;
    const long long plane = static_cast<long long>(W) * H;
    const long long planes = 3LL * count;
    // stream-ordered scratch (valid inside CUDA graph capture as well)
    float* lab = nullptr;
    double* rows = nullptr;
    CF_CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&lab), sizeof(float) * planes * plane, stream));
    CF_CUDA_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&rows), sizeof(double) * planes * plane, stream));
    rgb_to_lab(ctx, rgb, count, W, H, lab, stream);
    const long long nrows = planes * H;
    launch_on(ctx, stream, "lab_integral", dim3(static_cast<unsigned>((nrows + 127) / 128)), dim3(128), 0,
              prefix_rows_double_kernel, lab, rows, nrows, W);
    const long long ncols = planes * W;
    launch_on(ctx, stream, "lab_integral", dim3(static_cast<unsigned>((ncols + 127) / 128)), dim3(128), 0,
              prefix_cols_float_kernel, rows, color_out, planes, W, H);
    CF_CUDA_CHECK(cudaFreeAsync(rows, stream));
    CF_CUDA_CHECK(cudaFreeAsync(lab, stream));
}

}  // namespace cf

using namespace cf;

extern "C" {

cf_status cf_fill_depth(cf_context* ctx, int count, int width, int height, uint16_t* depth_mm, int device_pointers) {
    return guard([&] {
        CF_REQUIRE(ctx && depth_mm, "cf_fill_depth: NULL argument");
        CF_REQUIRE(count >= 1 && width >= 1 && height >= 1, "cf_fill_depth: empty input");
        make_current(ctx);
        const size_t bytes = sizeof(uint16_t) * count * static_cast<size_t>(width) * height;
        if (device_pointers) {
            fill_depth_frames(ctx, depth_mm, count, width, height, ctx->stream);
        } else {
            DevArray<uint16_t> d;
            d.reserve(bytes / 2);
            CF_CUDA_CHECK(cudaMemcpyAsync(d.get(), depth_mm, bytes, cudaMemcpyHostToDevice, ctx->stream));
            fill_depth_frames(ctx, d.get(), count, width, height, ctx->stream);
            CF_CUDA_CHECK(cudaMemcpyAsync(depth_mm, d.get(), bytes, cudaMemcpyDeviceToHost, ctx->stream));
        }
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_integrate_planes(cf_context* ctx, int count, int width, int height, const float* color,
                              const int32_t* depth, float* color_integral, int32_t* depth_integral,
                              int device_pointers) {
    return guard([&] {
        CF_REQUIRE(ctx && color && depth && color_integral && depth_integral, "cf_integrate_planes: NULL argument");
        CF_REQUIRE(count >= 1 && width >= 1 && height >= 1, "cf_integrate_planes: empty input");
        make_current(ctx);
        cudaStream_t st = ctx->stream;
        const long long plane = static_cast<long long>(width) * height;
        const long long cplanes = 3LL * count, dplanes = 2LL * count;
        DevArray<float> d_color;
        DevArray<double> rows;
        DevArray<float> d_cout;
        DevArray<int32_t> d_depth;
        rows.reserve(static_cast<size_t>(cplanes * plane));
        const float* c_in = color;
        float* c_out = color_integral;
        int32_t* dep = depth_integral;
        if (!device_pointers) {
            d_color.reserve(static_cast<size_t>(cplanes * plane));
            d_cout.reserve(static_cast<size_t>(cplanes * plane));
            d_depth.reserve(static_cast<size_t>(dplanes * plane));
            CF_CUDA_CHECK(cudaMemcpyAsync(d_color.get(), color, sizeof(float) * cplanes * plane, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(d_depth.get(), depth, sizeof(int32_t) * dplanes * plane, cudaMemcpyHostToDevice,
                                          st));
            c_in = d_color.get();
            c_out = d_cout.get();
            dep = d_depth.get();
        } else if (depth_integral != depth) {
            CF_CUDA_CHECK(cudaMemcpyAsync(depth_integral, depth, sizeof(int32_t) * dplanes * plane,
                                          cudaMemcpyDeviceToDevice, st));
        }
        const long long crows = cplanes * height, ccols = cplanes * width;
        launch(ctx, "integral_planes", dim3(static_cast<unsigned>((crows + 127) / 128)), dim3(128), 0,
               prefix_rows_double_kernel, c_in, rows.get(), crows, width);
        launch(ctx, "integral_planes", dim3(static_cast<unsigned>((ccols + 127) / 128)), dim3(128), 0,
               prefix_cols_float_kernel, rows.get(), c_out, cplanes, width, height);
        const long long drows = dplanes * height, dcols = dplanes * width;
        launch(ctx, "integral_planes", dim3(static_cast<unsigned>((drows + 127) / 128)), dim3(128), 0,
               prefix_rows_int_kernel, dep, drows, width);
        launch(ctx, "integral_planes", dim3(static_cast<unsigned>((dcols + 127) / 128)), dim3(128), 0,
               prefix_cols_int_kernel, dep, dplanes, width, height);
        if (!device_pointers) {
            CF_CUDA_CHECK(cudaMemcpyAsync(color_integral, c_out, sizeof(float) * cplanes * plane, cudaMemcpyDeviceToHost,
                                          st));
            CF_CUDA_CHECK(cudaMemcpyAsync(depth_integral, dep, sizeof(int32_t) * dplanes * plane, cudaMemcpyDeviceToHost,
                                          st));
        }
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
    });
}

cf_status cf_rgb_to_cielab(cf_context* ctx, int count, int width, int height, const uint8_t* rgb, float* lab,
                           int device_pointers) {
    return guard([&] {
        CF_REQUIRE(ctx && rgb && lab, "cf_rgb_to_cielab: NULL argument");
        CF_REQUIRE(count >= 1 && width >= 1 && height >= 1, "cf_rgb_to_cielab: empty input");
        make_current(ctx);
        const size_t px = count * static_cast<size_t>(width) * height;
        if (device_pointers) {
            rgb_to_lab(ctx, rgb, count, width, height, lab, ctx->stream);
        } else {
            DevArray<uint8_t> d_rgb;
            DevArray<float> d_lab;
            d_rgb.reserve(px * 3);
            d_lab.reserve(px * 3);
            CF_CUDA_CHECK(cudaMemcpyAsync(d_rgb.get(), rgb, px * 3, cudaMemcpyHostToDevice, ctx->stream));
            rgb_to_lab(ctx, d_rgb.get(), count, width, height, d_lab.get(), ctx->stream);
            CF_CUDA_CHECK(cudaMemcpyAsync(lab, d_lab.get(), px * 3 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        }
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

}  // extern "C"
