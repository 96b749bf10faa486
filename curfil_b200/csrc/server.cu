// Serving: continuous batching of dense per-pixel prediction on a forest resident on the device.
//
// Replaces the reference's per-image test loop (predict.cpp:209-375, one classifyImage launch and
// stream sync per tree per image, serialised by a global mutex). Requests are copied at submit and
// queued. A launcher thread forms batches from whatever is queued when a pipeline slot frees up:
// frames of any size are admitted while the slot's share of the device-memory budget holds them,
// copied host->device through pinned staging, integrated, and classified by ONE launch over all
// frames of the batch; results come back device->host on the same slot stream. Each slot has a waiter
// thread that publishes the slot's results as soon as its event completes, in whatever order the slots
// finish. With several slots, one batch's copies overlap another batch's kernels, and requests arriving
// during a launch join the next batch. With device priorities on, a batch holds frames of one size
// class and goes to the server's stream for that class (one stream per CUDA priority level, chosen by
// the frame's pixel count), so the thread blocks of small frames are dispatched ahead of a large
// frame's blocks that have not started yet, and batches of one class run in admission order.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "features.h"
#include "forest.h"

namespace cf {
namespace {

constexpr size_t kAlign = 256;
inline size_t up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Request {
    int64_t id = 0;
    int W = 0, H = 0;
    std::vector<uint8_t> rgb;
    std::vector<uint16_t> depth;
    std::vector<uint8_t> labels;
    std::vector<float> probs;
    double submit_ms = 0, admitted_ms = 0, done_ms = 0;
    int batch_id = -1, batch_frames = 0;
    bool done = false;
    cf_status status = CF_OK;
    std::string error;
};

// Bytes a frame occupies in a slot.
size_t frame_device_bytes(int W, int H, int C, bool probs) {
    const size_t px = static_cast<size_t>(W) * H;
    return up(px * 3) + up(px * 2) + up(px * 12) + up(px * 8) + up(px) + (probs ? up(px * 4 * C) : 0);
}
size_t frame_host_bytes(int W, int H, int C, bool probs) {
    const size_t px = static_cast<size_t>(W) * H;
    return up(px * 3) + up(px * 2) + up(px) + (probs ? up(px * 4 * C) : 0);
}

// Pixel count of the most urgent device-priority level (one 160x120 frame); each further level holds
// frames up to four times larger.
constexpr long long kUrgentPixels = 160 * 120;

// Device-priority level (size class) of a frame of `px` pixels among `levels` (0 most urgent).
int priority_level(long long px, int levels) {
    int b = 0;
    while (px > kUrgentPixels && b + 1 < levels) {
        px = (px + 3) / 4;
        b++;
    }
    return b;
}

struct Slot {
    // the streams this slot's batches may run on (not owned): its own stream, or with device priorities
    // the server's streams of each level, most urgent first, shared by all slots. A slot's buffers are
    // reused only after its previous batch's event has completed on the host, so no stream has to keep
    // one slot's batches in order.
    std::vector<cudaStream_t> streams;
    cudaStream_t stream = nullptr;       // the stream of the batch in flight
    cudaEvent_t done = nullptr;
    cudaEvent_t copied = nullptr;        // the batch's inputs are on the device (with a copy stream)
    DeviceBuffer dev;
    PinnedBuffer host;
    PinnedBuffer desc;                   // the batch's FrameDesc array, staged for the copy
    DevArray<FrameDesc> frames;
    std::vector<FrameDesc> h_frames;
    std::vector<std::shared_ptr<Request>> batch;
    std::vector<size_t> host_off;   // per frame: offset of rgb in host staging
    int batch_id = -1;
    bool busy = false;       // admitted a batch (set by the launcher, cleared when its results are out)
    bool launched = false;   // the batch's work is enqueued and `done` recorded behind it
    std::thread waiter;      // publishes this slot's batches as each completes, in any order across slots
};

}  // namespace
}  // namespace cf

using namespace cf;

struct cf_server {
    cf_forest* forest = nullptr;
    cf_context* ctx = nullptr;
    cf_server_config cfg{};
    size_t slot_bytes = 0, slot_host_bytes = 0;
    std::vector<std::unique_ptr<Slot>> slots;
    // Every stream the server created. With device priorities there is one stream per level, shared by
    // the slots: CUDA maps streams onto a few hardware queues (CUDA_DEVICE_MAX_CONNECTIONS, 8 by
    // default), and a stream for each slot and level would put a small batch in the same queue as, and
    // behind, a large one.
    std::vector<cudaStream_t> owned_streams;
    int levels = 1;                       // device-priority levels (1 without device priorities)
    cudaStream_t copy_stream = nullptr;   // host->device inputs of every batch (with device priorities)
    std::mutex mu;
    std::condition_variable cv_queue, cv_slot, cv_done, cv_inflight;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<int64_t, std::shared_ptr<Request>> requests;
    int64_t next_id = 1, submitted = 0, completed = 0, rejected = 0, batches = 0;
    int64_t expired = 0;   // rejected after waiting longer than max_queue_ms
    bool stopping = false;
    std::thread launcher;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::string fatal;

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }

    void launch_loop() {
        cudaSetDevice(ctx->device);
        int batch_id = 0;
        for (;;) {
            Slot* slot = nullptr;
            std::vector<std::shared_ptr<Request>> batch;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_queue.wait(lk, [&] { return stopping || !queue.empty(); });
                if (stopping && queue.empty()) return;
                cv_slot.wait(lk, [&] {
                    if (stopping) return true;
                    for (auto& s : slots)
                        if (!s->busy) return true;
                    return false;
                });
                if (stopping && queue.empty()) return;
                for (auto& s : slots)
                    if (!s->busy) {
                        slot = s.get();
                        break;
                    }
                if (!slot) continue;
                const double now = now_ms();
                // load shedding: a request still queued max_queue_ms after its submission is refused
                // instead of being served late (the queue is in arrival order, so expired requests are
                // at its front)
                if (cfg.max_queue_ms > 0.0f) {
                    while (!queue.empty() && now - queue.front()->submit_ms > cfg.max_queue_ms) {
                        auto& r = queue.front();
                        r->status = CF_ERR_REJECTED;
                        r->error = "request waited longer than max_queue_ms in the queue";
                        r->done_ms = now;
                        r->done = true;
                        rejected++;
                        expired++;
                        queue.pop_front();
                    }
                    cv_done.notify_all();
                    if (queue.empty()) continue;
                }
                // admission: frames in the policy's order (arrival, or smallest first with requests
                // older than max_wait_ms ahead) while they fit in the slot's budget
                size_t dev = 0, host = 0;
                int level = -1;   // with device priorities a batch holds frames of one size class
                while (!queue.empty() && static_cast<int>(batch.size()) < cfg.max_batch_frames) {
                    size_t pick = 0;
                    if (cfg.policy == 1 && now - queue.front()->submit_ms <= cfg.max_wait_ms) {
                        // the queue is in arrival order: the front is the oldest, so no request is overdue
                        for (size_t i = 1; i < queue.size(); i++)
                            if (static_cast<long long>(queue[i]->W) * queue[i]->H <
                                static_cast<long long>(queue[pick]->W) * queue[pick]->H)
                                pick = i;
                    }
                    auto r = queue[pick];
                    if (cfg.device_priority) {
                        const int l = priority_level(static_cast<long long>(r->W) * r->H, levels);
                        if (level >= 0 && l != level) break;
                        level = l;
                    }
                    const size_t d = frame_device_bytes(r->W, r->H, forest->C, cfg.return_probabilities != 0);
                    const size_t h = frame_host_bytes(r->W, r->H, forest->C, cfg.return_probabilities != 0);
                    if (dev + d > slot_bytes || host + h > slot_host_bytes) break;
                    dev += d;
                    host += h;
                    batch.push_back(r);
                    queue.erase(queue.begin() + static_cast<long>(pick));
                }
                if (batch.empty()) continue;
                slot->busy = true;
                const double t = now_ms();
                for (auto& r : batch) {
                    r->admitted_ms = t;
                    r->batch_id = batch_id;
                    r->batch_frames = static_cast<int>(batch.size());
                }
            }
            try {
                run_batch(slot, batch, batch_id);
            } catch (const std::exception& e) {
                // whatever was enqueued must finish before the slot's buffers are handed out again,
                // possibly to a batch on another of its streams
                if (copy_stream) cudaStreamSynchronize(copy_stream);
                if (slot->stream) cudaStreamSynchronize(slot->stream);
                std::lock_guard<std::mutex> lk(mu);
                for (auto& r : batch) {
                    r->status = CF_ERR_CUDA;
                    r->error = e.what();
                    r->done = true;
                }
                slot->batch.clear();
                slot->busy = false;
                cv_done.notify_all();
                cv_slot.notify_all();
                cv_inflight.notify_all();
                continue;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                slot->launched = true;
                batches++;
            }
            cv_inflight.notify_all();
            batch_id++;
        }
    }

    void run_batch(Slot* slot, std::vector<std::shared_ptr<Request>>& batch, int batch_id) {
        const int C = forest->C;
        const bool want_probs = cfg.return_probabilities != 0;
        char* dbase = static_cast<char*>(slot->dev.get());
        char* hbase = static_cast<char*>(slot->host.get());
        size_t doff = 0, hoff = 0;
        slot->h_frames.resize(batch.size());
        slot->host_off.resize(batch.size());
        slot->batch = batch;
        slot->batch_id = batch_id;
        // the size class of the batch's largest frame (with device priorities all its frames share one)
        long long frame_px = 0;
        for (auto& r : batch) frame_px = std::max(frame_px, static_cast<long long>(r->W) * r->H);
        slot->stream = slot->streams[priority_level(frame_px, static_cast<int>(slot->streams.size()))];
        // inputs go on the copy stream when there is one, so they do not queue behind the kernels
        // already waiting in the batch's (shared) priority stream
        cudaStream_t in = copy_stream ? copy_stream : slot->stream;
        struct Planes {
            const uint8_t* rgb;
            uint16_t* depth;
            float* color;
            int2* integral;
        };
        std::vector<Planes> planes(batch.size());
        int blocks = 0;
        for (size_t i = 0; i < batch.size(); i++) {
            Request& r = *batch[i];
            const size_t px = static_cast<size_t>(r.W) * r.H;
            uint8_t* d_rgb = reinterpret_cast<uint8_t*>(dbase + doff);
            doff += up(px * 3);
            uint16_t* d_depth = reinterpret_cast<uint16_t*>(dbase + doff);
            doff += up(px * 2);
            float* d_color = reinterpret_cast<float*>(dbase + doff);
            doff += up(px * 12);
            int2* d_int = reinterpret_cast<int2*>(dbase + doff);
            doff += up(px * 8);
            uint8_t* d_labels = reinterpret_cast<uint8_t*>(dbase + doff);
            doff += up(px);
            float* d_probs = nullptr;
            if (want_probs) {
                d_probs = reinterpret_cast<float*>(dbase + doff);
                doff += up(px * 4 * C);
            }
            slot->host_off[i] = hoff;
            uint8_t* h_rgb = reinterpret_cast<uint8_t*>(hbase + hoff);
            std::memcpy(h_rgb, r.rgb.data(), px * 3);
            hoff += up(px * 3);
            uint16_t* h_depth = reinterpret_cast<uint16_t*>(hbase + hoff);
            std::memcpy(h_depth, r.depth.data(), px * 2);
            hoff += up(px * 2);
            hoff += up(px) + (want_probs ? up(px * 4 * C) : 0);
            CF_CUDA_CHECK(cudaMemcpyAsync(d_rgb, h_rgb, px * 3, cudaMemcpyHostToDevice, in));
            CF_CUDA_CHECK(cudaMemcpyAsync(d_depth, h_depth, px * 2, cudaMemcpyHostToDevice, in));
            planes[i] = {d_rgb, d_depth, d_color, d_int};
            FrameDesc& fr = slot->h_frames[i];
            fr.color = d_color;
            fr.depth = d_int;
            fr.probs = d_probs;
            fr.labels = d_labels;
            fr.width = r.W;
            fr.height = r.H;
            fr.first_block = blocks;
            fr.pad = 0;
            blocks += classify_blocks_for(r.W, r.H);
        }
        // the descriptors go through pinned memory: a copy from pageable memory may wait for the stream
        std::memcpy(slot->desc.get(), slot->h_frames.data(), sizeof(FrameDesc) * batch.size());
        CF_CUDA_CHECK(cudaMemcpyAsync(slot->frames.get(), slot->desc.get(), sizeof(FrameDesc) * batch.size(),
                                      cudaMemcpyHostToDevice, in));
        if (in != slot->stream) {
            CF_CUDA_CHECK(cudaEventRecord(slot->copied, in));
            CF_CUDA_CHECK(cudaStreamWaitEvent(slot->stream, slot->copied, 0));
        }
        for (size_t i = 0; i < batch.size(); i++) {
            const Planes& pl = planes[i];
            integrate_frames(ctx, pl.rgb, pl.depth, 1, batch[i]->W, batch[i]->H, pl.color, pl.integral, slot->stream,
                             forest->preprocess);
        }
        classify_frames(ctx, forest, slot->frames.get(), static_cast<int>(batch.size()), blocks, slot->stream);
        for (size_t i = 0; i < batch.size(); i++) {
            Request& r = *batch[i];
            const size_t px = static_cast<size_t>(r.W) * r.H;
            char* h = hbase + slot->host_off[i] + up(px * 3) + up(px * 2);
            CF_CUDA_CHECK(cudaMemcpyAsync(h, slot->h_frames[i].labels, px, cudaMemcpyDeviceToHost, slot->stream));
            if (want_probs)
                CF_CUDA_CHECK(cudaMemcpyAsync(h + up(px), slot->h_frames[i].probs, px * 4 * C, cudaMemcpyDeviceToHost,
                                              slot->stream));
        }
        CF_CUDA_CHECK(cudaEventRecord(slot->done, slot->stream));
    }

    // One waiter per slot: a batch's results are published when its own event completes, so a small
    // batch that finishes first is not held behind a larger one launched before it.
    void complete_loop(Slot* slot) {
        cudaSetDevice(ctx->device);
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                // a busy slot that is not yet launched is between admission and enqueue: wait for it
                cv_inflight.wait(lk, [&] { return slot->launched || (stopping && !slot->busy); });
                if (!slot->launched) return;
            }
            const cudaError_t e = cudaEventSynchronize(slot->done);
            const double t = now_ms();
            const int C = forest->C;
            const bool want_probs = cfg.return_probabilities != 0;
            char* hbase = static_cast<char*>(slot->host.get());
            for (size_t i = 0; i < slot->batch.size(); i++) {
                Request& r = *slot->batch[i];
                if (e != cudaSuccess) {
                    r.status = CF_ERR_CUDA;
                    r.error = cudaGetErrorString(e);
                    continue;
                }
                const size_t px = static_cast<size_t>(r.W) * r.H;
                const char* h = hbase + slot->host_off[i] + up(px * 3) + up(px * 2);
                r.labels.assign(reinterpret_cast<const uint8_t*>(h), reinterpret_cast<const uint8_t*>(h) + px);
                if (want_probs)
                    r.probs.assign(reinterpret_cast<const float*>(h + up(px)),
                                   reinterpret_cast<const float*>(h + up(px)) + px * C);
                r.rgb.clear();
                r.rgb.shrink_to_fit();
                r.depth.clear();
                r.depth.shrink_to_fit();
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                for (auto& r : slot->batch) {
                    r->done_ms = t;
                    r->done = true;
                    completed++;
                }
                slot->batch.clear();
                slot->busy = false;
                slot->launched = false;
            }
            cv_done.notify_all();
            cv_slot.notify_all();
        }
    }
};

extern "C" {

cf_status cf_server_create(cf_forest* forest, const cf_server_config* config, cf_server** out) {
    return guard([&] {
        CF_REQUIRE(forest && config && out, "cf_server_create: NULL argument");
        CF_REQUIRE(config->hbm_budget_bytes > 0 && config->max_batch_frames >= 1 && config->max_pending >= 1 &&
                       config->pipeline_depth >= 1,
                   "cf_server_create: invalid configuration");
        CF_REQUIRE(config->policy == 0 || (config->policy == 1 && config->max_wait_ms > 0.0f),
                   "cf_server_create: policy is 0 (arrival order) or 1 (smallest first, max_wait_ms > 0)");
        CF_REQUIRE(config->device_priority == 0 || config->device_priority == 1,
                   "cf_server_create: device_priority is 0 or 1");
        CF_REQUIRE(config->max_queue_ms >= 0.0f, "cf_server_create: max_queue_ms must be >= 0 (0: no limit)");
        cf_context* ctx = forest->ctx;
        make_current(ctx);
        std::unique_ptr<cf_server> s(new cf_server());
        s->forest = forest;
        s->ctx = ctx;
        s->cfg = *config;
        s->slot_bytes = static_cast<size_t>(config->hbm_budget_bytes) / config->pipeline_depth;
        // host staging mirrors the device share (inputs and outputs only)
        s->slot_host_bytes = s->slot_bytes;
        // device-priority levels: greatest (most urgent) .. least, or the default priority alone
        int least = 0, greatest = 0;
        if (config->device_priority) CF_CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        std::vector<cudaStream_t> level_streams;
        for (int l = 0; config->device_priority && l <= least - greatest; l++) {
            cudaStream_t st = nullptr;
            CF_CUDA_CHECK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, greatest + l));
            s->owned_streams.push_back(st);
            level_streams.push_back(st);
        }
        if (config->device_priority) {
            s->levels = static_cast<int>(level_streams.size());
            CF_CUDA_CHECK(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
            s->owned_streams.push_back(s->copy_stream);
        }
        for (int i = 0; i < config->pipeline_depth; i++) {
            auto slot = std::make_unique<Slot>();
            if (config->device_priority) {
                slot->streams = level_streams;
            } else {
                cudaStream_t st = nullptr;
                CF_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                s->owned_streams.push_back(st);
                slot->streams.push_back(st);
            }
            slot->stream = slot->streams[0];
            CF_CUDA_CHECK(cudaEventCreateWithFlags(&slot->done, cudaEventDisableTiming));
            CF_CUDA_CHECK(cudaEventCreateWithFlags(&slot->copied, cudaEventDisableTiming));
            slot->dev.reserve(s->slot_bytes);
            slot->host.reserve(s->slot_host_bytes);
            slot->desc.reserve(sizeof(FrameDesc) * config->max_batch_frames);
            slot->frames.reserve(config->max_batch_frames);
            s->slots.push_back(std::move(slot));
        }
        cf_server* raw = s.get();
        for (auto& slot : s->slots) {
            Slot* sl = slot.get();
            sl->waiter = std::thread([raw, sl] { raw->complete_loop(sl); });
        }
        s->launcher = std::thread([raw] { raw->launch_loop(); });
        context_retain(ctx);
        *out = s.release();
    });
}

cf_status cf_server_destroy(cf_server* server) {
    return guard([&] {
        if (!server) return;
        {
            std::lock_guard<std::mutex> lk(server->mu);
            server->stopping = true;
            for (auto& r : server->queue) {
                r->status = CF_ERR_STATE;
                r->error = "server stopped";
                r->done = true;
            }
            server->queue.clear();
        }
        server->cv_queue.notify_all();
        server->cv_slot.notify_all();
        server->cv_inflight.notify_all();
        if (server->launcher.joinable()) server->launcher.join();
        // drain batches still on the device
        {
            std::unique_lock<std::mutex> lk(server->mu);
            server->cv_done.wait_for(lk, std::chrono::seconds(60), [&] {
                for (auto& s : server->slots)
                    if (s->busy) return false;
                return true;
            });
        }
        server->cv_inflight.notify_all();
        for (auto& s : server->slots)
            if (s->waiter.joinable()) s->waiter.join();
        cudaSetDevice(server->ctx->device);
        for (cudaStream_t st : server->owned_streams) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        for (auto& s : server->slots) {
            if (s->done) cudaEventDestroy(s->done);
            if (s->copied) cudaEventDestroy(s->copied);
        }
        cf_context* ctx = server->ctx;
        delete server;
        context_release(ctx);
    });
}

cf_status cf_server_submit(cf_server* server, int width, int height, const uint8_t* rgb, const uint16_t* depth_mm,
                           int64_t* request_id) {
    return guard([&] {
        CF_REQUIRE(server && rgb && depth_mm && request_id, "cf_server_submit: NULL argument");
        CF_REQUIRE(width >= 1 && height >= 1, "cf_server_submit: empty frame");
        const bool probs = server->cfg.return_probabilities != 0;
        if (frame_device_bytes(width, height, server->forest->C, probs) > server->slot_bytes ||
            frame_host_bytes(width, height, server->forest->C, probs) > server->slot_host_bytes) {
            std::lock_guard<std::mutex> lk(server->mu);
            server->rejected++;
            fail(CF_ERR_REJECTED, "frame larger than the per-batch memory budget");
        }
        auto r = std::make_shared<Request>();
        const size_t px = static_cast<size_t>(width) * height;
        r->W = width;
        r->H = height;
        r->rgb.assign(rgb, rgb + px * 3);
        r->depth.assign(depth_mm, depth_mm + px);
        {
            std::lock_guard<std::mutex> lk(server->mu);
            CF_REQUIRE(!server->stopping, "cf_server_submit: server is stopping");
            if (static_cast<int>(server->queue.size()) >= server->cfg.max_pending) {
                server->rejected++;
                fail(CF_ERR_REJECTED, "request queue is full");
            }
            r->id = server->next_id++;
            r->submit_ms = server->now_ms();
            server->queue.push_back(r);
            server->requests[r->id] = r;
            server->submitted++;
            *request_id = r->id;
        }
        server->cv_queue.notify_one();
    });
}

cf_status cf_server_wait(cf_server* server, int64_t request_id, double timeout_s, uint8_t* labels, float* probabilities,
                         cf_request_stats* stats) {
    return guard([&] {
        CF_REQUIRE(server, "cf_server_wait: server is NULL");
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(server->mu);
            auto it = server->requests.find(request_id);
            CF_REQUIRE(it != server->requests.end(), "cf_server_wait: unknown request id");
            r = it->second;
            const auto deadline = std::chrono::steady_clock::now() +
                                  std::chrono::microseconds(static_cast<int64_t>(std::max(0.0, timeout_s) * 1e6));
            if (!server->cv_done.wait_until(lk, deadline, [&] { return r->done; }))
                fail(CF_ERR_TIMEOUT, "cf_server_wait: request " + std::to_string(request_id) + " not done in time");
            server->requests.erase(it);
        }
        if (r->status != CF_OK) fail(r->status, r->error);
        if (labels) std::memcpy(labels, r->labels.data(), r->labels.size());
        if (probabilities) {
            CF_REQUIRE(!r->probs.empty(), "cf_server_wait: the server was created without probabilities");
            std::memcpy(probabilities, r->probs.data(), sizeof(float) * r->probs.size());
        }
        if (stats) {
            stats->submit_ms = r->submit_ms;
            stats->admitted_ms = r->admitted_ms;
            stats->done_ms = r->done_ms;
            stats->batch_id = r->batch_id;
            stats->batch_frames = r->batch_frames;
        }
    });
}

cf_status cf_server_counters(cf_server* server, int64_t* submitted, int64_t* completed, int64_t* rejected,
                             int64_t* batches) {
    return guard([&] {
        CF_REQUIRE(server, "cf_server_counters: server is NULL");
        std::lock_guard<std::mutex> lk(server->mu);
        if (submitted) *submitted = server->submitted;
        if (completed) *completed = server->completed;
        if (rejected) *rejected = server->rejected;
        if (batches) *batches = server->batches;
    });
}

}  // extern "C"
