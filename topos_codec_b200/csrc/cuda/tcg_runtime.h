// tcg_runtime.h - CUDA-side runtime shared by the encode and decode drivers:
// device selection, context leases (one stream + grow-only device/pinned
// buffers per concurrent caller), frozen device tables, error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <atomic>
#include <vector>

#include "../tcg_device.h"

#define TCG_OK 0
#define TCG_ERR_INVALID_ARGUMENT (-1)
#define TCG_ERR_OUT_OF_MEMORY (-2)
#define TCG_ERR_LIMIT_EXCEEDED (-8)
#define TCG_ERR_MALFORMED (-9)
#define TCG_ERR_TRUNCATED (-10)
#define TCG_ERR_CHECKSUM_MISMATCH (-11)
#define TCG_ERR_BUFFER_TOO_SMALL (-15)
#define TCG_ERR_NOT_IMPLEMENTED (-16)

namespace tcg {

// Grow-only device buffer.
struct DBuf {
    void* p = nullptr;
    size_t cap = 0;
};

// Grow-only pinned host buffer.
struct HBuf {
    void* p = nullptr;
    size_t cap = 0;
};

enum BufId {
    B_PIX, B_COEF, B_MASK, B_DCM, B_NOPS, B_OPOFF, B_HIST, B_STAB, B_OPS, B_STAGE,
    B_SRES, B_PKT, B_DESC, B_FRES, B_ALPHA, B_DEC_COEF, B_DEC_TAB, B_DEC_OUT, B_DEC_PKT,
    B_DEC_RES, B_TMP0, B_TMP1, B_SIZED_PIX, B_SIZED_PKT, B_UMAP, B_COUNT
};

// Kernel identities for optional per-kernel event timing.
enum KernelId {
    K_FDCT, K_TOKENS, K_SELECT, K_OPSCAN, K_OPGEN, K_CHAIN, K_ALPHA, K_PACK_SIZES, K_PACK_COPY, K_PACK_CRC,
    K_PACK_HEADER, K_DCRC, K_DTABLES, K_DCHAIN, K_DCHAIN_W, K_DIDCT, K_DALPHA, K_DALPHA_MED, K_DCONCEAL, K_DEBLOCK_V,
    K_DEBLOCK_H, K_WALK, K_DECIMATE, K_UNIT_MAP, K_COUNT
};

constexpr int MAX_PROF = 64;

struct Ctx {
    cudaStream_t stream = nullptr;
    // The second and third streams are created on first use (side_stream,
    // aux_stream): the streams of a process share a small set of hardware work
    // queues (8 unless CUDA_DEVICE_MAX_CONNECTIONS says otherwise), and two
    // streams on one queue can wait for each other's work, so a context holds
    // no stream it does not use and orders nothing on one it did not use.
    cudaStream_t side = nullptr;                  // second stream for work split across two launches
    cudaEvent_t fork = nullptr, join = nullptr;   // ordering between stream and side
    cudaStream_t aux = nullptr;                   // third stream for independent work (alpha planes)
    cudaEvent_t afork = nullptr, ajoin = nullptr; // ordering between stream and aux
    bool side_open = false, aux_open = false;     // work queued there since the last completed call
    cudaEvent_t gate = nullptr;                // recorded after a call's input copies (pipelined chunks)
    cudaEvent_t t0 = nullptr, t1 = nullptr;    // whole-call device time
    cudaEvent_t kev[2 * MAX_PROF] = {};        // per-kernel timing (profiling on)
    int kid[MAX_PROF] = {};
    int kn = 0;
    bool prof = false;
    DBuf d[B_COUNT];
    HBuf h[4];
    // pinned buffers outgrown by h[]: freeing pinned memory synchronises the
    // whole device, so they are freed only where the device is idle for this
    // context anyway (trim_idle, shutdown)
    std::vector<void*> h_retired;
    Ctx* next = nullptr;
    int cls = -1;  // lease class of the thread that last used it (tcg_set_lease_class)
};

// Call bracketing: records the device start/end events and, with profiling
// enabled, folds the per-kernel event pairs into the process totals.
void call_begin(Ctx* c);
void call_end(Ctx* c);  // after the stream was synchronised
void kern_begin(Ctx* c, int id);
void kern_end(Ctx* c);
void kern_begin_on(Ctx* c, int id, cudaStream_t s);  // timing events on another of the context's streams
void kern_end_on(Ctx* c, cudaStream_t s);

// Launch on the context's stream. With TCG_SYNC_EACH=1 in the environment
// every launch is followed by a stream synchronisation, so a failing kernel is
// named in the error instead of surfacing at a later call (diagnostics only).
#define TCG_LAUNCH(C, id, kern, grid, block, smem, ...)                 \
    do {                                                                 \
        tcg::kern_begin((C), (id));                                      \
        kern<<<(grid), (block), (smem), (C)->stream>>>(__VA_ARGS__);     \
        tcg::kern_end((C));                                              \
        tcg::note_launch(1);                                             \
        if (tcg::sync_each()) {                                          \
            cudaError_t le_ = cudaGetLastError();                        \
            if (le_ == cudaSuccess) { le_ = cudaStreamSynchronize((C)->stream); } \
            if (le_ != cudaSuccess) { return tcg::cuda_fail(le_, #kern); } \
        }                                                                \
    } while (0)

// The same on a given stream of the context.
#define TCG_LAUNCH_ON(C, strm, id, kern, grid, block, smem, ...)         \
    do {                                                                 \
        tcg::kern_begin_on((C), (id), (strm));                           \
        kern<<<(grid), (block), (smem), (strm)>>>(__VA_ARGS__);          \
        tcg::kern_end_on((C), (strm));                                   \
        tcg::note_launch(1);                                             \
        if (tcg::sync_each()) {                                          \
            cudaError_t le_ = cudaGetLastError();                        \
            if (le_ == cudaSuccess) { le_ = cudaStreamSynchronize(strm); } \
            if (le_ != cudaSuccess) { return tcg::cuda_fail(le_, #kern); } \
        }                                                                \
    } while (0)

// Host-memory batches are coded as up to PIPE_MAX_CHUNKS chunks, each on its
// own context: chunk i's input copies wait for chunk i-1's (an event), so the
// copies of later chunks overlap the kernels of earlier ones and each chunk's
// results go back while later chunks still compute. The frame ranges split the
// batch's copy bytes evenly. pipeline_plan returns the chunk count (1 = code
// the batch in one piece, at most PIPE_ENCODE_CHUNKS or PIPE_DECODE_CHUNKS)
// and fills starts[0..k]. TCG_PIPELINE=<n> in the environment forces n chunks
// (0 or 1: never pipeline; at most PIPE_MAX_CHUNKS).
//
// Decode stops at three chunks: the chunks' entropy chains run side by side,
// and with four chunks of a 60-frame 3840x2160 batch their single-warp blocks
// land unevenly on the SM sub-partitions, so every chain slows (per 60 frames:
// 3 chunks 134-138 ms, 4 chunks 167-180 ms, one piece 161 ms). The encode
// chain packs 32 slices per warp and keeps gaining up to four (114 ms; one
// piece 150 ms).
constexpr uint32_t PIPE_MAX_CHUNKS = 4;
constexpr uint32_t PIPE_ENCODE_CHUNKS = 4;
constexpr uint32_t PIPE_DECODE_CHUNKS = 3;
uint32_t pipeline_plan(bool decode, const uint64_t* frame_bytes, uint32_t count, uint32_t* starts);
bool host_memory(const void* p);  // pinned or pageable host memory (not device or managed)
void set_last_ms(double ms);      // device time reported by tcg_last_ms for this thread's last call
// Device time between two completed events of this device (0 on error).
double event_span_ms(cudaEvent_t a, cudaEvent_t b);

// The context's second / third stream, created on first use, with the call's
// pending-work flag set (call_begin of the next call orders that work before
// its own when this call fails before rejoining it). nullptr (error set) when
// the stream cannot be created.
cudaStream_t side_stream(Ctx* c);
cudaStream_t aux_stream(Ctx* c);

// Lease a context (creates one when none is free). Thread-safe.
Ctx* ctx_acquire();
void ctx_release(Ctx* c);

// Ensure device buffer capacity; returns false (and sets the error) on failure.
bool dreserve(Ctx* c, BufId id, size_t bytes);
// Frees the device buffers of every idle (pooled) context.
void trim_idle();
bool hreserve(Ctx* c, int id, size_t bytes);

template <typename T>
T* dptr(Ctx* c, BufId id) { return static_cast<T*>(c->d[id].p); }

// Device-global frozen tables (defined in tcg_runtime.cu, uploaded by init).
struct DevTables {
    const uint32_t* div_m;   // [4097] rANS division magic (index = freq)
    const uint8_t* div_l;    // [4097] shift
    const double* log2;      // [4097] exact log2 series values
    const uint32_t* crc;     // [8][256] slicing-by-8 CRC-32 tables
    const uint32_t* qscale;  // [2][96] classic / refined qp scale
};
const DevTables& tables();

bool ensure_init();
void note_launch(uint32_t n = 1);
// true when TCG_SYNC_EACH=1 was set in the environment at first use
bool sync_each();

// CUDA error -> host status + thread-local detail.
int32_t cuda_fail(cudaError_t e, const char* what);

// Host-side helpers for CRC combination (GF(2) polynomial arithmetic).
uint32_t crc_shift_op(uint64_t len_bytes);

}  // namespace tcg

#define TCG_CHECK(call)                                           \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) { return tcg::cuda_fail(e_, #call); } \
    } while (0)
