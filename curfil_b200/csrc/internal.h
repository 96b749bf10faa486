// Internal host-side definitions shared by the curfil_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <atomic>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/curfil_b200.h"

namespace cf {

struct Error : std::runtime_error {
    cf_status code;
    Error(cf_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(cf_status code, const std::string& msg) { throw Error(code, msg); }

#define CF_CUDA_CHECK(x)                                                                           \
    do {                                                                                           \
        cudaError_t e__ = (x);                                                                     \
        if (e__ != cudaSuccess)                                                                    \
            ::cf::fail(e__ == cudaErrorMemoryAllocation ? CF_ERR_OOM : CF_ERR_CUDA,                \
                       std::string(#x) + ": " + cudaGetErrorString(e__));                          \
    } while (0)

#define CF_REQUIRE(cond, msg)                                                                      \
    do {                                                                                           \
        if (!(cond)) ::cf::fail(CF_ERR_INVALID, msg);                                              \
    } while (0)

void set_last_error(const std::string& msg);

// Runs f and converts exceptions into a status code plus the thread's last-error message.
template <class F>
cf_status guard(F&& f) {
    try {
        f();
        return CF_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc& e) {
        set_last_error(std::string("host allocation failed: ") + e.what());
        return CF_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return CF_ERR_INVALID;
    }
}

// Owning device allocation (cudaMalloc); grows, never shrinks.
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) {
        o.ptr_ = nullptr;
        o.bytes_ = 0;
    }
    ~DeviceBuffer() { release(); }
    void reserve(size_t bytes) {
        if (bytes <= bytes_) return;
        release();
        if (bytes == 0) return;
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            fail(CF_ERR_OOM, "cudaMalloc(" + std::to_string(bytes) + ") failed: " + cudaGetErrorString(e));
        }
        ptr_ = p;
        bytes_ = bytes;
    }
    void release() {
        if (ptr_) cudaFree(ptr_);
        ptr_ = nullptr;
        bytes_ = 0;
    }
    void* get() const { return ptr_; }
    size_t bytes() const { return bytes_; }

private:
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
};

template <class T>
class DevArray {
public:
    void reserve(size_t n) { buf_.reserve(n * sizeof(T)); }
    T* get() const { return static_cast<T*>(buf_.get()); }
    size_t capacity() const { return buf_.bytes() / sizeof(T); }
    void release() { buf_.release(); }

private:
    DeviceBuffer buf_;
};

// Pinned host staging buffer (cudaHostAlloc); grows, never shrinks.
class PinnedBuffer {
public:
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    ~PinnedBuffer() {
        if (ptr_) cudaFreeHost(ptr_);
    }
    void reserve(size_t bytes) {
        if (bytes <= bytes_) return;
        if (ptr_) cudaFreeHost(ptr_);
        ptr_ = nullptr;
        bytes_ = 0;
        CF_CUDA_CHECK(cudaHostAlloc(&ptr_, bytes, cudaHostAllocDefault));
        bytes_ = bytes;
    }
    void* get() const { return ptr_; }

private:
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
};

}  // namespace cf

struct cf_context {
    int device = 0;
    int num_sms = 0;
    size_t smem_per_block_optin = 0;
    size_t l2_bytes = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    bool timing = false;
    std::atomic<int64_t> launches{0};
    // objects (datasets, forests, servers) holding this context; destruction waits for the last
    std::atomic<int> refs{0};
    std::atomic<bool> closed{false};
    cf_eval_tuning tuning = default_tuning();   // split-search launch shape
    // the tree-training buffers of a destroyed dataset, kept for the next dataset that trains on this
    // context (cf_forest_train makes a dataset per call; the buffers grow level by level otherwise)
    void* spare_trainer = nullptr;
    void (*spare_trainer_free)(void*) = nullptr;

    // measured on B200 with 200 frames 640x480, 40 classes, 2000 features x 20 thresholds: a 28 KB
    // histogram leaves ~140 KB of the SM's unified memory to L1 for the integral-image gathers; sample
    // groups without increment aggregation were 8 % faster than thread-per-sample with aggregation.
    // With 1000 frames and 4000 features x 32 thresholds, tiles of at most 16 features (shared staging
    // sized for 16, not 32) left more L1 and were 3-12 % faster per level. Up to 2048 items per CTA
    // slot of at least 16 K evaluations, in multiples of 4 features, were 4-21 % faster on the levels
    // of that workload (more CTAs on one node's samples at a time, sharing their gathers in L2).
    static cf_eval_tuning default_tuning() { return cf_eval_tuning{16, 7168, 0, 3, 4, 2048.0f, 1, 16384, 1, 8192, 1}; }
    std::mutex mu;
    struct KernelEvents {
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
        double total_ms = 0.0;
        int64_t count = 0;
    };
    std::map<std::string, KernelEvents> kernel_events;
    std::vector<cudaEvent_t> event_pool;

    cudaEvent_t take_event();
    void collect_events();
};

namespace cf {

// Records CUDA events around one launch on the context stream when timing is enabled.
class LaunchScope {
public:
    LaunchScope(cf_context* ctx, cudaStream_t stream, const char* name);
    ~LaunchScope() noexcept(false);

private:
    cf_context* ctx_;
    cudaStream_t stream_;
    const char* name_;
    cudaEvent_t start_ = nullptr;
};

template <class Kernel, class... Args>
inline void launch_on(cf_context* ctx, cudaStream_t stream, const char* name, dim3 grid, dim3 block, size_t smem,
                      Kernel kernel, Args... args) {
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return;
    LaunchScope scope(ctx, stream, name);
    kernel<<<grid, block, smem, stream>>>(args...);
    CF_CUDA_CHECK(cudaGetLastError());
    ctx->launches++;
}

template <class Kernel, class... Args>
inline void launch(cf_context* ctx, const char* name, dim3 grid, dim3 block, size_t smem, Kernel kernel,
                   Args... args) {
    launch_on(ctx, ctx->stream, name, grid, block, smem, kernel, args...);
}

inline void make_current(cf_context* ctx) { CF_CUDA_CHECK(cudaSetDevice(ctx->device)); }

// A closed context is freed when the last object using it is destroyed.
void context_retain(cf_context* ctx);
void context_release(cf_context* ctx);

}  // namespace cf

struct cf_dataset {
    cf_context* ctx = nullptr;
    int n = 0, width = 0, height = 0;
    cf::DevArray<float> color;   // [n][3][H][W] integral, float
    cf::DevArray<int2> depth;    // [n][H][W] integral {depth mm sum (wrapping int32), valid count}
    cf::DevArray<uint8_t> raw_rgb;      // upload staging
    cf::DevArray<uint16_t> raw_depth;
    // tree-training buffers reused across cf_train_tree calls on this dataset (grow-only)
    void* trainer = nullptr;
    void (*trainer_free)(void*) = nullptr;
    ~cf_dataset() {
        if (trainer && trainer_free) trainer_free(trainer);
    }
};
