// tc_server.cpp - continuous-batching request server over the batched frame
// calls (extension; the reference has no server).
//
// Requests (encode or decode of one frame, caller-owned buffers in host or
// device memory) enter two queues. Each direction has a pool of workers, each
// coding through its own call context (its own CUDA stream): an idle worker
// takes the requests that have arrived - an even share of them when other
// workers are idle too, at most max_batch_frames - and codes them in one
// batched call. Requests that arrive while batches run are picked up by the
// next idle worker at once, so their work overlaps the batches already on the
// GPU instead of waiting for them. Half of each direction's workers take
// frames up to 2560x1440 only, the others larger frames first, so small
// requests always have a worker of their own. Admission: a batch takes requests while
// the estimated device bytes of everything in flight fit the server's budget
// and the device's free memory (the first request of a batch always goes, so
// one large request cannot stall the queue). The free memory is read once,
// when the server starts: querying it while requests run (cudaMemGetInfo and
// the pool's counters) stalled calls in flight for up to a second, and with
// the queries gone the V8 stream's p99 fell from 100-700 ms to under 5 ms.
// Each direction's workers lease their own contexts, so a context holds one
// direction's buffers and all of them fit in the memory mapped at start. A
// worker that finds fewer than four V7-R2 requests waits up to 4 ms for
// more (a V7-R2 batch costs its longest slice chain whatever its size); V8
// requests go at once. V8 decodes run through the
// single-frame V8 decoder (the batched decode takes V7 packets only, as the
// reference's does). Each request's latency is measured from submission to
// completion.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

extern "C" {
#include "../tcg_device.h"
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
    bool big = false;    // above BIG_PIXELS luma samples
    bool v8 = false;     // decode of a V8 packet
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
    std::deque<Request> q[2][2];  // [encode][big]
    std::unordered_map<uint64_t, Result> done;
    uint64_t next_ticket = 1;
    uint64_t budget = 0;
    uint64_t inflight = 0;       // estimated device bytes of the batches running
    uint32_t max_frames = 64;
    uint32_t idle[2][2] = {{0, 0}, {0, 0}};  // idle workers [encode][lane: 0 small frames only, 1 any]
    uint64_t free0 = UINT64_MAX;        // device memory free (with the pool's unused part) at creation
    uint64_t batch_bytes = UINT64_MAX;  // estimated device bytes of one batch at most
    bool stop = false;
    std::vector<std::thread> workers;
    int device = 0;
};

namespace {

// frames above this many luma samples (past 2560x1440) are served by the
// general workers only
constexpr uint64_t BIG_PIXELS = 2560ull * 1440ull;

// device bytes one frame of w x h luma samples needs while it is coded, with
// the buffers' growth margin: per 8x8 block of a 4:2:2 frame (two blocks per
// 64 luma samples) encode holds 128 B of samples, 256 B of coefficients,
// 12 B of mask and DC, 1 KB of operation words, 512 B of staging and the
// packet; decode the packet, 256 B of coefficients, 128 B of planes and the
// slice tables
uint64_t frame_bytes(uint32_t w, uint32_t h, bool encode)
{
    const uint64_t px = (uint64_t)w * h;
    return encode ? px * 84u + (1u << 20) : px * 20u + (1u << 20);
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
        // V7 packets in one batched call, V8 packets one by one
        std::vector<uint32_t> v7;
        for (uint32_t i = 0; i < n; ++i) {
            if (!batch[i].v8) {
                v7.push_back(i);
                continue;
            }
            res[i].status = tc_frame_decode(pk[i].data, pk[i].size, &planes[(size_t)i * TC_FRAME_MAX_PLANES],
                                            &strides[(size_t)i * TC_FRAME_MAX_PLANES], &res[i].info);
        }
        if (!v7.empty()) {
            const uint32_t m = (uint32_t)v7.size();
            std::vector<topos_batch_packet> pk7(m);
            std::vector<uint16_t*> pl7((size_t)m * TC_FRAME_MAX_PLANES);
            std::vector<size_t> st7((size_t)m * TC_FRAME_MAX_PLANES);
            for (uint32_t k = 0; k < m; ++k) {
                pk7[k] = pk[v7[k]];
                for (uint32_t p = 0; p < TC_FRAME_MAX_PLANES; ++p) {
                    pl7[(size_t)k * TC_FRAME_MAX_PLANES + p] = planes[(size_t)v7[k] * TC_FRAME_MAX_PLANES + p];
                    st7[(size_t)k * TC_FRAME_MAX_PLANES + p] = strides[(size_t)v7[k] * TC_FRAME_MAX_PLANES + p];
                }
            }
            const int32_t rc = tc_frame_decode_batch(pk7.data(), m, pl7.data(), st7.data(), infos.data());
            for (uint32_t k = 0; k < m; ++k) {
                Result& r = res[v7[k]];
                r.info = infos[k];
                r.status = rc < 0 ? rc : (infos[k].concealed_slices != 0 ? TC_WARN_CONCEALED : TC_OK);
            }
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

// A worker of lane 0 takes small frames only; a worker of lane 1 takes large
// frames first and small ones when no large frame waits. So small requests
// never queue behind a batch of large frames while a lane-0 worker is free.
void worker(tcg_server* s, bool encode, int lane)
{
    cudaSetDevice(s->device);
    tcg_set_lease_class(encode ? 1 : 0);  // a context keeps one direction's buffers
    std::deque<Request>* qs = s->q[encode ? 1 : 0];
    uint32_t* idle = s->idle[encode ? 1 : 0];
    auto has_work = [&] { return !qs[0].empty() || (lane == 1 && !qs[1].empty()); };
    for (;;) {
        std::vector<Request> batch;
        uint64_t used = 0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            idle[lane]++;
            s->cv_work.wait(lk, [&] { return s->stop || has_work(); });
            idle[lane]--;
            if (s->stop && !has_work()) { return; }
        }
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (!has_work()) { continue; }  // another worker took them meanwhile
            const bool big = lane == 1 && !qs[1].empty();
            std::deque<Request>& q = qs[big ? 1 : 0];
            {
                // a V7-R2 batch costs its longest slice chain whatever its
                // size: give a lone V7-R2 request a few milliseconds of company
                const Request& f = q.front();
                const bool v7 = f.encode ? f.cfg.reserved[0] != 9u : !f.v8;
                if (v7 && q.size() < 4u && !s->stop) {
                    const size_t n0 = q.size();
                    s->cv_work.wait_for(lk, std::chrono::milliseconds(4),
                                        [&] { return s->stop || q.size() >= 4u || q.size() < n0; });
                    if (q.empty()) { continue; }
                }
            }
            // an even share of what has arrived when other workers that can
            // take it are idle too
            const uint32_t others = big ? idle[1] : idle[0] + idle[1];
            const size_t share = (q.size() + others) / (others + 1u);
            const size_t take = std::min<size_t>(std::max<size_t>(share, 1u), s->max_frames);
            // the batches in flight against the budget and against 7/8 of the
            // memory that was free when the server started
            const uint64_t room = s->budget > s->inflight ? s->budget - s->inflight : 0u;
            const uint64_t mem = s->free0 - s->free0 / 8u;
            const uint64_t cap = std::min<uint64_t>(room, mem > s->inflight ? mem - s->inflight : 0u);
            while (!q.empty() && batch.size() < take) {
                const uint64_t b = q.front().bytes;
                if (!batch.empty() && (used + b > cap || used + b > s->batch_bytes)) { break; }
                used += b;
                batch.push_back(q.front());
                q.pop_front();
            }
            s->inflight += used;
            if (!qs[0].empty() || !qs[1].empty()) { s->cv_work.notify_all(); }  // more for the next idle worker
        }
        run_batch(s, batch, encode);
        std::lock_guard<std::mutex> g(s->mu);
        s->inflight -= used;
        if (!qs[0].empty() || !qs[1].empty()) { s->cv_work.notify_all(); }
    }
}

uint64_t submit(tcg_server* s, Request&& r, bool encode)
{
    std::lock_guard<std::mutex> g(s->mu);
    r.ticket = s->next_ticket++;
    r.encode = encode;
    r.t_submit = Clock::now();
    const uint64_t t = r.ticket;
    s->q[encode ? 1 : 0][r.big ? 1 : 0].push_back(std::move(r));
    s->cv_work.notify_all();
    return t;
}

}  // namespace

extern "C" {

TC_EXPORT int32_t tcg_server_create(uint64_t max_bytes_in_flight, uint32_t max_batch_frames, tcg_server** out)
{
    return tcg_server_create_ex(max_bytes_in_flight, max_batch_frames, 4u, out);
}

TC_EXPORT int32_t tcg_server_create_ex(uint64_t max_bytes_in_flight, uint32_t max_batch_frames, uint32_t workers,
                                       tcg_server** out)
{
    if (out == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_create: out is NULL"); }
    *out = NULL;
    if (max_batch_frames == 0u || max_batch_frames > TC_BATCH_MAX_FRAMES) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_create: max_batch_frames %u outside 1..%u",
                       max_batch_frames, (unsigned)TC_BATCH_MAX_FRAMES);
    }
    if (workers == 0u || workers > 16u) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "tcg_server_create: workers %u outside 1..16", workers);
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
    {
        // map memory for the workers' buffers now: a call that grows its
        // buffers while others run would otherwise map new memory, and that
        // stalled the device for up to 0.6 s under a V8 request stream
        uint64_t fr = 0, tot = 0;
        tcg_mem_info(&fr, &tot);
        if (fr != 0u) { s->free0 = fr; }
        const uint64_t want = std::min<uint64_t>(fr / 2u, 64ull << 30);
        if (want > (1ull << 30) && tcg_pool_reserve(want) == 0) {
            // every worker's context keeps its largest batch's buffers (and a
            // context serves either direction), so batches are sized for all
            // of them to fit in what was mapped
            s->batch_bytes = want / (3u * workers);
        }
    }
    // half of each direction's workers (rounded down) serve small frames only
    for (uint32_t i = 0; i < workers; ++i) {
        const int lane = i < workers / 2u ? 0 : 1;
        s->workers.emplace_back(worker, s, true, lane);
        s->workers.emplace_back(worker, s, false, lane);
    }
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
    for (std::thread& t : s->workers) { t.join(); }
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
    r.big = (uint64_t)cfg->visible_width * cfg->visible_height > BIG_PIXELS;
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
    r.big = (uint64_t)info.visible_width * info.visible_height > BIG_PIXELS;
    r.v8 = tc_packet_major(packet, size) == 8;
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
