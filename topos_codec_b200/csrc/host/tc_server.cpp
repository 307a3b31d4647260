// tc_server.cpp - continuous-batching request server over the batched frame
// calls (extension; the reference has no server).
//
// Requests (encode or decode of one frame, caller-owned buffers in host or
// device memory) enter two queues. One worker per direction takes every
// request that has arrived, up to a frame count and a byte budget, and codes
// them in one batched call; requests that arrive meanwhile wait for the next
// batch. The two workers run at the same time on their own call contexts
// (their own CUDA streams), so encode and decode batches overlap on the GPU.
// Admission: a batch only takes requests while the estimated device bytes of
// the batch fit both the server's budget and the device's free memory.
// Each request's latency is measured from submission to completion.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

extern "C" {
#include "tc_internal.h"
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    bool encode = true;
    // encode
    topos_frame_config cfg{};
    topos_frame_input input{};
    uint8_t* out = nullptr;
    size_t out_cap = 0;
    // decode
    const uint8_t* packet = nullptr;
    size_t size = 0;
    uint16_t* planes[TC_FRAME_MAX_PLANES] = {nullptr, nullptr, nullptr, nullptr};
    size_t strides[TC_FRAME_MAX_PLANES] = {0, 0, 0, 0};
    uint64_t bytes = 0;  // estimated device footprint
    Clock::time_point t_submit;
};

struct Result {
    int32_t status = 0;
    topos_frame_stats stats{};
    topos_frame_output info{};
    double latency_ms = 0.0;
};

}  // namespace

struct tcg_server {
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> q_enc, q_dec;
    std::unordered_map<uint64_t, Result> done;
    uint64_t next_ticket = 1;
    uint64_t budget = 0;
    uint32_t max_frames = 64;
    bool stop = false;
    std::thread w_enc, w_dec;
    int device = 0;
};

namespace {

// device bytes one frame of w x h luma samples needs while it is coded
// (samples, coefficients, operation words, staging, packet for encode;
// packet, coefficients, tables, planes for decode), rounded up
uint64_t frame_bytes(uint32_t w, uint32_t h, bool encode)
{
    const uint64_t px = (uint64_t)w * h;
    return encode ? px * 40u + (1u << 20) : px * 20u + (1u << 20);
}

uint64_t device_free()
{
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return fr;
}

void run_batch(tcg_server* s, std::vector<Request>& batch, bool encode)
{
    const uint32_t n = (uint32_t)batch.size();
    std::vector<Result> res(n);
    if (encode) {
        std::vector<topos_frame_config> cfgs(n);
        std::vector<topos_frame_input> ins(n);
        std::vector<uint8_t*> outs(n);
        std::vector<size_t> caps(n);
        std::vector<topos_frame_stats> stats(n);
        std::vector<int32_t> rcs(n, 0);
        for (uint32_t i = 0; i < n; ++i) {
            cfgs[i] = batch[i].cfg;
            ins[i] = batch[i].input;
            outs[i] = batch[i].out;
            caps[i] = batch[i].out_cap;
        }
        const int32_t rc = tcg_frame_encode_batch(cfgs.data(), ins.data(), n, outs.data(), caps.data(), stats.data(),
                                                  rcs.data());
        for (uint32_t i = 0; i < n; ++i) {
            res[i].status = rc < 0 && rcs[i] == 0 ? rc : rcs[i];
            res[i].stats = stats[i];
        }
    } else {
        std::vector<topos_batch_packet> pk(n);
        std::vector<uint16_t*> planes((size_t)n * TC_FRAME_MAX_PLANES);
        std::vector<size_t> strides((size_t)n * TC_FRAME_MAX_PLANES);
        std::vector<topos_frame_output> infos(n);
        for (uint32_t i = 0; i < n; ++i) {
            pk[i].data = batch[i].packet;
            pk[i].size = batch[i].size;
            for (uint32_t p = 0; p < TC_FRAME_MAX_PLANES; ++p) {
                planes[(size_t)i * TC_FRAME_MAX_PLANES + p] = batch[i].planes[p];
                strides[(size_t)i * TC_FRAME_MAX_PLANES + p] = batch[i].strides[p];
            }
        }
        const int32_t rc = tc_frame_decode_batch(pk.data(), n, planes.data(), strides.data(), infos.data());
        for (uint32_t i = 0; i < n; ++i) {
            res[i].info = infos[i];
            res[i].status = rc < 0 ? rc : (infos[i].concealed_slices != 0 ? TC_WARN_CONCEALED : TC_OK);
        }
    }
    const Clock::time_point t_end = Clock::now();
    std::lock_guard<std::mutex> g(s->mu);
    for (uint32_t i = 0; i < n; ++i) {
        res[i].latency_ms = std::chrono::duration<double, std::milli>(t_end - batch[i].t_submit).count();
        s->done[batch[i].ticket] = res[i];
    }
    s->cv_done.notify_all();
}

void worker(tcg_server* s, bool encode)
{
    cudaSetDevice(s->device);
    std::deque<Request>& q = encode ? s->q_enc : s->q_dec;
    for (;;) {
        std::vector<Request> batch;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !q.empty(); });
            if (s->stop && q.empty()) { return; }
            const uint64_t free_b = device_free();
            const uint64_t cap = free_b == 0 ? s->budget : std::min<uint64_t>(s->budget, free_b - free_b / 8);
            uint64_t used = 0;
            while (!q.empty() && batch.size() < s->max_frames) {
                const uint64_t b = q.front().bytes;
                // the first request always goes, so an oversized one cannot stall the queue
                if (!batch.empty() && used + b > cap) { break; }
                used += b;
                batch.push_back(q.front());
                q.pop_front();
            }
        }
        run_batch(s, batch, encode);
    }
}

uint64_t submit(tcg_server* s, Request&& r, bool encode)
{
    std::lock_guard<std::mutex> g(s->mu);
    r.ticket = s->next_ticket++;
    r.encode = encode;
    r.t_submit = Clock::now();
    const uint64_t t = r.ticket;
    (encode ? s->q_enc : s->q_dec).push_back(std::move(r));
    s->cv_work.notify_all();
    return t;
}

}  // namespace

extern "C" {

TC_EXPORT int32_t tcg_server_create(uint64_t max_bytes_in_flight, uint32_t max_batch_frames, tcg_server** out)
{
    if (out == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_create: out is NULL"); }
    *out = NULL;
    if (max_batch_frames == 0u || max_batch_frames > TC_BATCH_MAX_FRAMES) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_create: max_batch_frames %u outside 1..%u",
                       max_batch_frames, (unsigned)TC_BATCH_MAX_FRAMES);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return tc_fail(TC_ERR_NOT_IMPLEMENTED, "tcg_server_create: no CUDA device");
    }
    tcg_server* s = new (std::nothrow) tcg_server();
    if (s == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "tcg_server_create"); }
    s->budget = max_bytes_in_flight == 0u ? UINT64_MAX : max_bytes_in_flight;
    s->max_frames = max_batch_frames;
    s->device = dev;
    s->w_enc = std::thread(worker, s, true);
    s->w_dec = std::thread(worker, s, false);
    *out = s;
    return TC_OK;
}

TC_EXPORT void tcg_server_destroy(tcg_server* s)
{
    if (s == NULL) { return; }
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    s->w_enc.join();
    s->w_dec.join();
    delete s;
}

TC_EXPORT int32_t tcg_server_submit_encode(tcg_server* s, const topos_frame_config* cfg, const topos_frame_input* input,
                                           uint8_t* out, size_t out_cap, uint64_t* ticket)
{
    if (s == NULL || cfg == NULL || input == NULL || ticket == NULL) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_submit_encode: NULL argument");
    }
    Request r;
    r.cfg = *cfg;
    r.input = *input;
    r.out = out;
    r.out_cap = out_cap;
    r.bytes = frame_bytes(cfg->visible_width, cfg->visible_height, true);
    *ticket = submit(s, std::move(r), true);
    return TC_OK;
}

TC_EXPORT int32_t tcg_server_submit_decode(tcg_server* s, const uint8_t* packet, size_t size,
                                           uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                                           const size_t strides[TC_FRAME_MAX_PLANES], uint64_t* ticket)
{
    if (s == NULL || packet == NULL || planes_out == NULL || ticket == NULL) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_submit_decode: NULL argument");
    }
    // validate alone first, so one bad packet cannot fail a whole batch
    topos_frame_output info;
    const int32_t rc = tc_frame_decode(packet, size, NULL, NULL, &info);
    if (rc != TC_OK) { return rc; }
    Request r;
    r.packet = packet;
    r.size = size;
    for (uint32_t p = 0; p < TC_FRAME_MAX_PLANES; ++p) {
        r.planes[p] = planes_out[p];
        r.strides[p] = strides != NULL ? strides[p] : 0u;
    }
    r.bytes = frame_bytes(info.visible_width, info.visible_height, false);
    *ticket = submit(s, std::move(r), false);
    return TC_OK;
}

TC_EXPORT int32_t tcg_server_wait(tcg_server* s, uint64_t ticket, int32_t* status, topos_frame_stats* stats,
                                  topos_frame_output* info, double* latency_ms)
{
    if (s == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_wait: NULL server"); }
    std::unique_lock<std::mutex> lk(s->mu);
    if (ticket == 0u || ticket >= s->next_ticket) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_wait: unknown ticket %llu", (unsigned long long)ticket);
    }
    s->cv_done.wait(lk, [&] { return s->done.count(ticket) != 0u; });
    const Result r = s->done[ticket];
    s->done.erase(ticket);
    lk.unlock();
    if (status != NULL) { *status = r.status; }
    if (stats != NULL) { *stats = r.stats; }
    if (info != NULL) { *info = r.info; }
    if (latency_ms != NULL) { *latency_ms = r.latency_ms; }
    return TC_OK;
}

}  // extern "C"
