// Context, error reporting and per-kernel CUDA-event timing.
#include <cstring>

#include "internal.h"

namespace cf {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

void destroy_context_now(cf_context* ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->kernel_events)
        for (auto& pr : kv.second.pending) {
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    if (ctx->spare_trainer && ctx->spare_trainer_free) ctx->spare_trainer_free(ctx->spare_trainer);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

void context_retain(cf_context* ctx) { ctx->refs++; }

void context_release(cf_context* ctx) {
    if (--ctx->refs == 0 && ctx->closed.load()) destroy_context_now(ctx);
}

LaunchScope::LaunchScope(cf_context* ctx, cudaStream_t stream, const char* name)
    : ctx_(ctx), stream_(stream), name_(name) {
    if (ctx_->timing) {
        // launches recorded into a CUDA graph are not timed one by one
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CF_CUDA_CHECK(cudaStreamIsCapturing(stream_, &cs));
        if (cs != cudaStreamCaptureStatusNone) return;
        std::lock_guard<std::mutex> lock(ctx_->mu);
        start_ = ctx_->take_event();
        CF_CUDA_CHECK(cudaEventRecord(start_, stream_));
    }
}

LaunchScope::~LaunchScope() noexcept(false) {
    if (start_ == nullptr) return;
    std::lock_guard<std::mutex> lock(ctx_->mu);
    cudaEvent_t stop = ctx_->take_event();
    cudaEventRecord(stop, stream_);
    ctx_->kernel_events[name_].pending.emplace_back(start_, stop);
}

}  // namespace cf

cudaEvent_t cf_context::take_event() {
    if (!event_pool.empty()) {
        cudaEvent_t e = event_pool.back();
        event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    CF_CUDA_CHECK(cudaEventCreate(&e));
    return e;
}

void cf_context::collect_events() {
    for (auto& kv : kernel_events) {
        for (auto& pr : kv.second.pending) {
            CF_CUDA_CHECK(cudaEventSynchronize(pr.second));
            float ms = 0;
            CF_CUDA_CHECK(cudaEventElapsedTime(&ms, pr.first, pr.second));
            kv.second.total_ms += ms;
            kv.second.count++;
            event_pool.push_back(pr.first);
            event_pool.push_back(pr.second);
        }
        kv.second.pending.clear();
    }
}

extern "C" {

const char* cf_version(void) { return "curfil_b200 0.1 (sm_100a)"; }

size_t cf_last_error(char* buffer, size_t length) {
    const std::string& m = cf::g_last_error;
    if (buffer && length > 0) {
        const size_t n = m.size() < length - 1 ? m.size() : length - 1;
        std::memcpy(buffer, m.data(), n);
        buffer[n] = '\0';
    }
    return m.size();
}

cf_status cf_context_create(int device, cf_context** out) {
    return cf::guard([&] {
        CF_REQUIRE(out != nullptr, "cf_context_create: out is NULL");
        int count = 0;
        CF_CUDA_CHECK(cudaGetDeviceCount(&count));
        CF_REQUIRE(device >= 0 && device < count, "cf_context_create: no CUDA device " + std::to_string(device));
        CF_CUDA_CHECK(cudaSetDevice(device));
        cudaDeviceProp prop;
        CF_CUDA_CHECK(cudaGetDeviceProperties(&prop, device));
        CF_REQUIRE(prop.major >= 10, std::string("curfil_b200 needs an sm_100 device, found ") + prop.name);
        auto* ctx = new cf_context();
        ctx->device = device;
        ctx->num_sms = prop.multiProcessorCount;
        ctx->smem_per_block_optin = prop.sharedMemPerBlockOptin;
        ctx->l2_bytes = static_cast<size_t>(prop.l2CacheSize);
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete ctx;
            cf::fail(CF_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
        }
        ctx->stream = ctx->own_stream;
        *out = ctx;
    });
}

cf_status cf_context_destroy(cf_context* ctx) {
    return cf::guard([&] {
        if (!ctx) return;
        ctx->closed = true;
        if (ctx->refs.load() == 0) cf::destroy_context_now(ctx);
    });
}

cf_status cf_context_set_stream(cf_context* ctx, void* stream) {
    return cf::guard([&] {
        CF_REQUIRE(ctx, "cf_context_set_stream: ctx is NULL");
        ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    });
}

cf_status cf_context_synchronize(cf_context* ctx) {
    return cf::guard([&] {
        CF_REQUIRE(ctx, "cf_context_synchronize: ctx is NULL");
        cf::make_current(ctx);
        CF_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    });
}

cf_status cf_context_set_timing(cf_context* ctx, int enable) {
    return cf::guard([&] {
        CF_REQUIRE(ctx, "cf_context_set_timing: ctx is NULL");
        ctx->timing = enable != 0;
    });
}

cf_status cf_context_kernel_time(cf_context* ctx, const char* kernel, double* total_ms, int64_t* launches) {
    return cf::guard([&] {
        CF_REQUIRE(ctx && kernel, "cf_context_kernel_time: NULL argument");
        cf::make_current(ctx);
        std::lock_guard<std::mutex> lock(ctx->mu);
        ctx->collect_events();
        double ms = 0;
        int64_t n = 0;
        if (std::strcmp(kernel, "*") == 0) {
            for (auto& kv : ctx->kernel_events) {
                ms += kv.second.total_ms;
                n += kv.second.count;
            }
        } else {
            auto it = ctx->kernel_events.find(kernel);
            if (it != ctx->kernel_events.end()) {
                ms = it->second.total_ms;
                n = it->second.count;
            }
        }
        if (total_ms) *total_ms = ms;
        if (launches) *launches = n;
    });
}

cf_status cf_context_reset_timing(cf_context* ctx) {
    return cf::guard([&] {
        CF_REQUIRE(ctx, "cf_context_reset_timing: ctx is NULL");
        cf::make_current(ctx);
        std::lock_guard<std::mutex> lock(ctx->mu);
        ctx->collect_events();
        for (auto& kv : ctx->kernel_events) {
            kv.second.total_ms = 0;
            kv.second.count = 0;
        }
    });
}

int64_t cf_context_launch_count(cf_context* ctx) { return ctx ? ctx->launches.load() : 0; }

cf_status cf_context_device(cf_context* ctx, char* name, size_t name_length, int* num_sms, int* cc_major,
                            int* cc_minor) {
    return cf::guard([&] {
        CF_REQUIRE(ctx, "cf_context_device: ctx is NULL");
        cudaDeviceProp prop;
        CF_CUDA_CHECK(cudaGetDeviceProperties(&prop, ctx->device));
        if (name && name_length > 0) {
            std::strncpy(name, prop.name, name_length - 1);
            name[name_length - 1] = '\0';
        }
        if (num_sms) *num_sms = prop.multiProcessorCount;
        if (cc_major) *cc_major = prop.major;
        if (cc_minor) *cc_minor = prop.minor;
    });
}

cf_status cf_context_get_tuning(cf_context* ctx, cf_eval_tuning* out) {
    return cf::guard([&] {
        CF_REQUIRE(ctx && out, "cf_context_get_tuning: NULL argument");
        std::lock_guard<std::mutex> lock(ctx->mu);
        *out = ctx->tuning;
    });
}

cf_status cf_context_set_tuning(cf_context* ctx, const cf_eval_tuning* tuning) {
    return cf::guard([&] {
        CF_REQUIRE(ctx, "cf_context_set_tuning: ctx is NULL");
        const cf_eval_tuning t = tuning ? *tuning : cf_context::default_tuning();
        CF_REQUIRE(t.features_per_tile >= 2 && t.features_per_tile <= 64,
                   "cf_context_set_tuning: features_per_tile must be in [2, 64]");
        CF_REQUIRE(t.bins_budget_words >= 1024 && t.bins_budget_words <= 49152,
                   "cf_context_set_tuning: bins_budget_words must be in [1024, 49152]");
        CF_REQUIRE(t.warp_aggregate == 0 || t.warp_aggregate == 1, "cf_context_set_tuning: warp_aggregate is 0 or 1");
        CF_REQUIRE(t.ctas_per_sm >= 1 && t.ctas_per_sm <= 4, "cf_context_set_tuning: ctas_per_sm must be in [1, 4]");
        CF_REQUIRE(t.feature_granule >= 1 && t.feature_granule <= 64,
                   "cf_context_set_tuning: feature_granule must be in [1, 64]");
        CF_REQUIRE(t.items_per_slot > 0.0f && t.items_per_slot <= 8192.0f,
                   "cf_context_set_tuning: items_per_slot must be in (0, 8192]");
        CF_REQUIRE(t.sample_groups == 0 || t.sample_groups == 1, "cf_context_set_tuning: sample_groups is 0 or 1");
        CF_REQUIRE(t.min_item_evals >= 256 && t.min_item_evals <= (1 << 30),
                   "cf_context_set_tuning: min_item_evals must be in [256, 2^30]");
        CF_REQUIRE(t.stage_bins >= 0 && t.stage_bins <= 2, "cf_context_set_tuning: stage_bins must be 0, 1 or 2");
        CF_REQUIRE(t.stage_max_mb >= 1 && t.stage_max_mb <= 65536,
                   "cf_context_set_tuning: stage_max_mb must be in [1, 65536]");
        CF_REQUIRE(t.sample_order >= 0 && t.sample_order <= 2, "cf_context_set_tuning: sample_order must be 0, 1 or 2");
        std::lock_guard<std::mutex> lock(ctx->mu);
        ctx->tuning = t;
    });
}

}  // extern "C"
