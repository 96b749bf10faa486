// Evaluation helpers (predict.cpp:45-207): pixel accuracy with and without void labels and the
// confusion matrix, on the device; ConfusionMatrix::normalize / averageClassAccuracy on the host.
//
// calculatePixelAccuracy (predict.cpp:148-207): a pixel whose ground-truth label is ignored is
// skipped unless includeVoid; the accuracy is correct / (all pixels of the image when includeVoid,
// else correct + wrong); the confusion matrix [label][prediction] counts the pixels not skipped.
#include <vector>

#include "internal.h"

namespace cf {

namespace {

__global__ void accuracy_kernel(const uint8_t* __restrict__ pred, const uint8_t* __restrict__ truth, long long n, int C,
                                const uint8_t* __restrict__ ignored, int include_void,
                                unsigned long long* __restrict__ counts, unsigned long long* __restrict__ confusion,
                                int* __restrict__ bad) {
    extern __shared__ unsigned int s_conf[];   // [C][C] when it fits, else unused
    __shared__ unsigned long long s_correct, s_wrong;
    const bool local = C <= 64;
    if (threadIdx.x == 0) s_correct = s_wrong = 0ull;
    if (local)
        for (int i = threadIdx.x; i < C * C; i += blockDim.x) s_conf[i] = 0u;
    __syncthreads();
    unsigned int correct = 0, wrong = 0;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int label = truth[i], p = pred[i];
        if (label >= C || p >= C) {
            *bad = 1;
            continue;
        }
        if (!include_void && ignored[label]) continue;
        if (p == label) correct++;
        else wrong++;
        if (local) atomicAdd(&s_conf[label * C + p], 1u);
        else atomicAdd(&confusion[label * C + p], 1ull);
    }
    atomicAdd(&s_correct, static_cast<unsigned long long>(correct));
    atomicAdd(&s_wrong, static_cast<unsigned long long>(wrong));
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&counts[0], s_correct);
        atomicAdd(&counts[1], s_wrong);
    }
    if (local)
        for (int i = threadIdx.x; i < C * C; i += blockDim.x)
            if (s_conf[i]) atomicAdd(&confusion[i], static_cast<unsigned long long>(s_conf[i]));
}

}  // namespace

}  // namespace cf

using namespace cf;

extern "C" {

cf_status cf_pixel_accuracy(cf_context* ctx, int count, int width, int height, const uint8_t* prediction,
                            const uint8_t* ground_truth, int num_classes, const uint8_t* ignored, int include_void,
                            uint64_t* confusion, double* accuracy, int device_pointers) {
    return guard([&] {
        CF_REQUIRE(ctx && prediction && ground_truth && accuracy, "cf_pixel_accuracy: NULL argument");
        CF_REQUIRE(count >= 1 && width >= 1 && height >= 1, "cf_pixel_accuracy: empty input");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_pixel_accuracy: classes must be in [1, 256]");
        make_current(ctx);
        cudaStream_t st = ctx->stream;
        const int C = num_classes;
        const long long n = static_cast<long long>(count) * width * height;
        std::vector<uint8_t> ign(C, 0);
        if (ignored)
            for (int c = 0; c < C; c++) ign[c] = ignored[c] ? 1 : 0;
        DevArray<uint8_t> d_ign;
        DevArray<unsigned long long> d_counts, d_conf;
        DevArray<int> d_bad;
        DevArray<uint8_t> d_frames;
        if (!device_pointers) {
            d_frames.reserve(static_cast<size_t>(2 * n));
            CF_CUDA_CHECK(cudaMemcpyAsync(d_frames.get(), prediction, n, cudaMemcpyHostToDevice, st));
            CF_CUDA_CHECK(cudaMemcpyAsync(d_frames.get() + n, ground_truth, n, cudaMemcpyHostToDevice, st));
            prediction = d_frames.get();
            ground_truth = d_frames.get() + n;
        }
        d_ign.reserve(C);
        d_counts.reserve(2);
        d_conf.reserve(static_cast<size_t>(C) * C);
        d_bad.reserve(1);
        CF_CUDA_CHECK(cudaMemcpyAsync(d_ign.get(), ign.data(), C, cudaMemcpyHostToDevice, st));
        CF_CUDA_CHECK(cudaMemsetAsync(d_counts.get(), 0, 2 * sizeof(unsigned long long), st));
        CF_CUDA_CHECK(cudaMemsetAsync(d_conf.get(), 0, sizeof(unsigned long long) * C * C, st));
        CF_CUDA_CHECK(cudaMemsetAsync(d_bad.get(), 0, sizeof(int), st));
        const size_t smem = C <= 64 ? sizeof(unsigned int) * C * C : 0;
        const int grid = static_cast<int>(std::min<long long>(ctx->num_sms * 8LL, (n + 255) / 256));
        launch(ctx, "pixel_accuracy", dim3(grid), dim3(256), smem, accuracy_kernel, prediction, ground_truth, n, C,
               d_ign.get(), include_void, d_counts.get(), d_conf.get(), d_bad.get());
        unsigned long long counts[2];
        int bad = 0;
        std::vector<unsigned long long> conf(static_cast<size_t>(C) * C);
        CF_CUDA_CHECK(cudaMemcpyAsync(counts, d_counts.get(), sizeof(counts), cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(&bad, d_bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaMemcpyAsync(conf.data(), d_conf.get(), sizeof(unsigned long long) * C * C,
                                      cudaMemcpyDeviceToHost, st));
        CF_CUDA_CHECK(cudaStreamSynchronize(st));
        CF_REQUIRE(!bad, "cf_pixel_accuracy: a label or prediction >= number of classes");
        const double pixels = include_void ? static_cast<double>(n) : static_cast<double>(counts[0] + counts[1]);
        *accuracy = pixels > 0 ? static_cast<double>(counts[0]) / pixels : 0.0;
        if (confusion)
            for (size_t i = 0; i < conf.size(); i++) confusion[i] += conf[i];
    });
}

cf_status cf_confusion_average_class_accuracy(int num_classes, const uint64_t* confusion, const uint8_t* ignored,
                                              int include_void, double* normalized, double* average) {
    return guard([&] {
        CF_REQUIRE(confusion && average, "cf_confusion_average_class_accuracy: NULL argument");
        CF_REQUIRE(num_classes >= 1 && num_classes <= 256, "cf_confusion_average_class_accuracy: classes");
        const int C = num_classes;
        std::vector<double> m(static_cast<size_t>(C) * C);
        for (int l = 0; l < C; l++) {   // ConfusionMatrix::normalize: rows by their sums, empty rows stay 0
            double sum = 0.0;
            for (int p = 0; p < C; p++) sum += static_cast<double>(confusion[l * C + p]);
            for (int p = 0; p < C; p++)
                m[l * C + p] = sum == 0.0 ? static_cast<double>(confusion[l * C + p]) : confusion[l * C + p] / sum;
        }
        double total = 0.0;
        int n = 0;
        for (int l = 0; l < C; l++) {   // averageClassAccuracy: the diagonal, void classes left out unless asked
            if (!include_void && ignored && ignored[l]) continue;
            total += m[l * C + l];
            n++;
        }
        *average = n ? total / n : 0.0;
        if (normalized) std::copy(m.begin(), m.end(), normalized);
    });
}

}  // extern "C"
