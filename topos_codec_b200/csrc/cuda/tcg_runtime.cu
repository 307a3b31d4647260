// tcg_runtime.cu - device init, context leases, frozen tables.
#include <stdlib.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "tcg_runtime.h"

namespace tcg {

static std::mutex g_mu;
static Ctx* g_free = nullptr;
static bool g_init = false;
static int g_device = -1;
static DevTables g_tab;
// Stream-ordered pool for the call contexts' grow-only buffers. Growing a
// buffer frees and allocates in the order of the context's own stream, so it
// never synchronises the device (cudaMalloc / cudaFree do, and with several
// calls in flight - the request server's workers - that stalls all of them).
// The pool keeps what is freed (the release threshold at its maximum), so a
// context that grows reuses memory another context gave up instead of mapping
// new memory (with a 2 GB threshold a serving trace made 113 allocations in
// 15 s and its p99 latency rose from 137 to 928 ms); trim_idle returns idle
// contexts' buffers and the pool's free memory to the device.
static cudaMemPool_t g_pool = nullptr;
static constexpr uint64_t POOL_KEEP = ~0ull;
static std::atomic<uint64_t> g_launches{0};
static std::atomic<uint64_t> g_allocs{0};  // device and pinned host allocations made
static std::atomic<int> g_prof_on{0};
static double g_prof_ms[K_COUNT];
static uint64_t g_prof_n[K_COUNT];
static thread_local double t_last_ms = 0.0;
static const char* k_names[K_COUNT] = {
    "k_fdct", "k_tokens", "k_select", "k_opscan", "k_opgen", "k_chain", "k_alpha", "k_pack_sizes", "k_pack_copy",
    "k_pack_crc", "k_pack_header", "k_dcrc", "k_dtables", "k_dchain", "k_dchain_w", "k_didct", "k_dalpha", "k_dalpha_med",
    "k_dconceal", "k_deblock_v", "k_deblock_h", "k_walk", "k_decimate", "k_unit_map"};

void note_launch(uint32_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

bool sync_each()
{
    static const bool on = [] {
        const char* v = getenv("TCG_SYNC_EACH");
        return v != nullptr && v[0] == '1';
    }();
    return on;
}

void call_begin(Ctx* c)
{
    c->prof = g_prof_on.load(std::memory_order_relaxed) != 0;
    c->kn = 0;
    // work a failed earlier call may have left on the context's other streams
    // comes before this call's work
    if (c->side_open) {
        cudaEventRecord(c->join, c->side);
        cudaStreamWaitEvent(c->stream, c->join, 0);
    }
    if (c->aux_open) {
        cudaEventRecord(c->ajoin, c->aux);
        cudaStreamWaitEvent(c->stream, c->ajoin, 0);
    }
    cudaEventRecord(c->t0, c->stream);
}

static cudaStream_t open_stream(cudaStream_t* s, cudaEvent_t* fork, cudaEvent_t* join, bool* open)
{
    // events first: the stream exists only with both of them
    if ((*fork == nullptr && cudaEventCreateWithFlags(fork, cudaEventDisableTiming) != cudaSuccess) ||
        (*join == nullptr && cudaEventCreateWithFlags(join, cudaEventDisableTiming) != cudaSuccess)) {
        tcg_host_set_error(TCG_ERR_OUT_OF_MEMORY, "event creation failed");
        return nullptr;
    }
    if (*s == nullptr && cudaStreamCreateWithFlags(s, cudaStreamNonBlocking) != cudaSuccess) {
        *s = nullptr;
        tcg_host_set_error(TCG_ERR_OUT_OF_MEMORY, "stream creation failed");
        return nullptr;
    }
    *open = true;
    return *s;
}

cudaStream_t side_stream(Ctx* c) { return open_stream(&c->side, &c->fork, &c->join, &c->side_open); }
cudaStream_t aux_stream(Ctx* c) { return open_stream(&c->aux, &c->afork, &c->ajoin, &c->aux_open); }

void kern_begin(Ctx* c, int id)
{
    if (!c->prof || c->kn >= MAX_PROF) { return; }
    c->kid[c->kn] = id;
    cudaEventRecord(c->kev[2 * c->kn], c->stream);
}

void kern_end(Ctx* c)
{
    if (!c->prof || c->kn >= MAX_PROF) { return; }
    cudaEventRecord(c->kev[2 * c->kn + 1], c->stream);
    c->kn++;
}

void kern_begin_on(Ctx* c, int id, cudaStream_t s)
{
    if (!c->prof || c->kn >= MAX_PROF) { return; }
    c->kid[c->kn] = id;
    cudaEventRecord(c->kev[2 * c->kn], s);
}

void kern_end_on(Ctx* c, cudaStream_t s)
{
    if (!c->prof || c->kn >= MAX_PROF) { return; }
    cudaEventRecord(c->kev[2 * c->kn + 1], s);
    c->kn++;
}

// A batch is pipelined when its host copies total at least 256 MB (about 5 ms
// of PCIe time), with one chunk per 64 MB up to PIPE_MAX_CHUNKS.
constexpr uint64_t PIPE_MIN_BYTES = 256ull << 20;
constexpr uint64_t PIPE_CHUNK_BYTES = 64ull << 20;

uint32_t pipeline_plan(bool decode, const uint64_t* frame_bytes, uint32_t count, uint32_t* starts)
{
    const char* env = getenv("TCG_PIPELINE");
    const int forced = env != nullptr && env[0] != '\0' ? atoi(env) : -1;
    uint64_t total = 0;
    for (uint32_t f = 0; f < count; ++f) { total += frame_bytes[f]; }
    uint64_t k = 1;
    if (forced >= 0) {
        k = forced < 1 ? 1u : (uint64_t)forced;
    } else if (total >= PIPE_MIN_BYTES) {
        k = std::min<uint64_t>(total / PIPE_CHUNK_BYTES, decode ? PIPE_DECODE_CHUNKS : PIPE_ENCODE_CHUNKS);
    }
    k = std::min<uint64_t>(std::min<uint64_t>(k, PIPE_MAX_CHUNKS), count);
    k = k < 1u ? 1u : k;
    // chunk j-1 = [starts[j-1], starts[j]) takes frames until its share of the
    // bytes is reached, keeping at least one frame for each later chunk
    uint32_t f = 0;
    uint64_t acc = 0;
    starts[0] = 0;
    for (uint32_t j = 1; j < (uint32_t)k; ++j) {
        const uint64_t target = total / k * j;
        do { acc += frame_bytes[f++]; } while (f < count - ((uint32_t)k - j) && acc < target);
        starts[j] = f;
    }
    starts[k] = count;
    return (uint32_t)k;
}

bool host_memory(const void* p)
{
    if (p == nullptr) { return false; }
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeUnregistered;
}

double event_span_ms(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? (double)ms : 0.0;
}

void set_last_ms(double ms) { t_last_ms = ms; }

void call_end(Ctx* c)
{
    cudaEventRecord(c->t1, c->stream);
    cudaEventSynchronize(c->t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    t_last_ms = ms;
    // a completed call rejoined its other streams before its last work
    c->side_open = false;
    c->aux_open = false;
    if (c->prof && c->kn > 0) {
        std::lock_guard<std::mutex> lk(g_mu);
        for (int i = 0; i < c->kn; ++i) {
            float k = 0.f;
            cudaEventElapsedTime(&k, c->kev[2 * i], c->kev[2 * i + 1]);
            g_prof_ms[c->kid[i]] += k;
            g_prof_n[c->kid[i]] += 1;
        }
    }
    c->kn = 0;
}

int32_t cuda_fail(cudaError_t e, const char* what)
{
    char buf[200];
    snprintf(buf, sizeof(buf), "CUDA error %s in %s", cudaGetErrorString(e), what);
    const int32_t st = (e == cudaErrorMemoryAllocation) ? TCG_ERR_OUT_OF_MEMORY : TCG_ERR_INVALID_ARGUMENT;
    tcg_host_set_error(st, buf);
    return st;
}

// rANS division magic: q = umulhi(2x, m) >> l equals floor(x / f) for every
// x < 2^31 and 1 <= f <= 4096, with l = ceil(log2 f), m = ceil(2^(31+l) / f)
// (m < 2^32 for all such f).
static void build_div(uint32_t* m, uint8_t* l)
{
    m[0] = 0; l[0] = 0;
    for (uint32_t f = 1; f <= 4096u; ++f) {
        uint32_t s = 0;
        while ((1u << s) < f) { ++s; }
        const uint64_t num = (uint64_t)1 << (31u + s);
        m[f] = (uint32_t)((num + f - 1u) / f);
        l[f] = (uint8_t)s;
    }
}

static void build_crc(uint32_t* t)
{
    for (uint32_t i = 0; i < 256u; ++i) {
        uint32_t c = i;
        for (int k = 0; k < 8; ++k) { c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1; }
        t[i] = c;
    }
    for (uint32_t i = 0; i < 256u; ++i) {
        for (int s = 1; s < 8; ++s) { t[s * 256 + i] = (t[(s - 1) * 256 + i] >> 8) ^ t[t[(s - 1) * 256 + i] & 0xFFu]; }
    }
}

// qp scale tables (bitstream constants; classic and refined variants)
static const uint32_t k_scale[96] = {
    1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5, 6, 7,
    8, 10, 11, 13, 16, 19, 23, 27, 32, 38, 45, 54, 64, 76, 91, 108,
    128, 152, 181, 215, 256, 304, 362, 431, 512, 609, 724, 861, 1024, 1218, 1448, 1722,
    2048, 2435, 2896, 3444, 4096, 4871, 5793, 6889, 8192, 9742, 11585, 13777, 16384, 19484, 23170, 27555,
    32768, 38968, 46341, 55109, 65536, 77936, 92682, 110218,
    131072, 155872, 185364, 220436, 262144, 311744, 370728, 440872,
    524288, 623487, 741455, 881744, 1048576, 1246974, 1482910, 1763488,
    2097152, 2493948, 2965821, 3526975, 4194304, 4987896, 5931642, 7053950};
static const uint32_t k_scale_refined_hi[32] = {
    32768, 36781, 41285, 46341, 52016, 58386, 65536, 73562,
    82570, 92682, 104032, 116772, 131072, 147123, 165140, 185364,
    208064, 233544, 262144, 294247, 330281, 370728, 416128, 467088,
    524288, 588493, 660561, 741455, 832255, 934175, 1048576, 1176987};

static bool init_locked(int device)
{
    if (g_init) { return true; }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        tcg_host_set_error(TCG_ERR_NOT_IMPLEMENTED, "no CUDA device available: the GPU library has no CPU path");
        return false;
    }
    if (device < 0) {
        if (cudaGetDevice(&device) != cudaSuccess) { device = 0; }
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        tcg_host_set_error(TCG_ERR_INVALID_ARGUMENT, "cudaSetDevice failed");
        return false;
    }
    g_device = device;
    // every section starts on a 16-byte boundary (the log2 table holds doubles)
    auto a16 = [](size_t v) { return (v + 15u) & ~(size_t)15u; };
    const size_t om = 0, ol = a16(om + 4097 * 4), olg = a16(ol + 4097), oc = a16(olg + 4097 * 8),
                 oq = a16(oc + 8 * 256 * 4), bytes = a16(oq + 2 * 96 * 4);
    uint8_t* h = (uint8_t*)calloc(1, bytes);
    uint8_t* d = nullptr;
    if (h == nullptr || cudaMalloc(&d, bytes) != cudaSuccess) {
        free(h);
        tcg_host_set_error(TCG_ERR_OUT_OF_MEMORY, "device table allocation failed");
        return false;
    }
    g_allocs.fetch_add(1, std::memory_order_relaxed);
    uint32_t* m = (uint32_t*)(h + om);
    uint8_t* l = h + ol;
    double* lg = (double*)(h + olg);
    uint32_t* crc = (uint32_t*)(h + oc);
    uint32_t* qs = (uint32_t*)(h + oq);
    build_div(m, l);
    memcpy(lg, tc_log2_table(), 4097 * sizeof(double));
    build_crc(crc);
    for (int q = 0; q < 96; ++q) {
        qs[q] = k_scale[q];
        qs[96 + q] = q >= 64 ? k_scale_refined_hi[q - 64] : k_scale[q];
    }
    e = cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice);
    free(h);
    if (e != cudaSuccess) {
        cuda_fail(e, "table upload");
        return false;
    }
    {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if (cudaMemPoolCreate(&g_pool, &props) != cudaSuccess) {
            cudaGetLastError();
            tcg_host_set_error(TCG_ERR_OUT_OF_MEMORY, "device memory pool creation failed");
            return false;
        }
        uint64_t keep = POOL_KEEP;
        cudaMemPoolSetAttribute(g_pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    g_tab.div_m = (const uint32_t*)(d + om);
    g_tab.div_l = d + ol;
    g_tab.log2 = (const double*)(d + olg);
    g_tab.crc = (const uint32_t*)(d + oc);
    g_tab.qscale = (const uint32_t*)(d + oq);
    g_init = true;
    return true;
}

bool ensure_init()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!init_locked(-1)) { return false; }
    // Device selection is per host thread in the CUDA runtime.
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != g_device) { cudaSetDevice(g_device); }
    return true;
}

const DevTables& tables() { return g_tab; }

// A thread with a lease class (the request server's workers: one class per
// direction) takes an idle context of its class when there is one, so a
// context keeps the buffers of one kind of work; other threads take the most
// recently released context.
static thread_local int t_lease_class = -1;

Ctx* ctx_acquire()
{
    if (!ensure_init()) { return nullptr; }
    {
        std::lock_guard<std::mutex> lk(g_mu);
        Ctx** link = nullptr;
        if (t_lease_class < 0) {
            link = &g_free;
        } else {
            Ctx** unclassed = nullptr;
            for (Ctx** l = &g_free; *l != nullptr; l = &(*l)->next) {
                if ((*l)->cls == t_lease_class) {
                    link = l;
                    break;
                }
                if ((*l)->cls < 0 && unclassed == nullptr) { unclassed = l; }
            }
            if (link == nullptr) { link = unclassed; }
        }
        if (link != nullptr && *link != nullptr) {
            Ctx* c = *link;
            *link = c->next;
            c->next = nullptr;
            c->cls = t_lease_class;
            return c;
        }
    }
    Ctx* c = new Ctx();
    c->cls = t_lease_class;
    bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->gate, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreate(&c->t0) == cudaSuccess && cudaEventCreate(&c->t1) == cudaSuccess;
    for (int i = 0; ok && i < 2 * MAX_PROF; ++i) { ok = cudaEventCreate(&c->kev[i]) == cudaSuccess; }
    if (!ok) {
        tcg_host_set_error(TCG_ERR_OUT_OF_MEMORY, "stream creation failed");
        delete c;
        return nullptr;
    }
    return c;
}

void ctx_release(Ctx* c)
{
    if (c == nullptr) { return; }
    std::lock_guard<std::mutex> lk(g_mu);
    c->next = g_free;
    g_free = c;
}

// Frees the device buffers of every context in the free pool (their streams
// first run dry); the next call on such a context allocates again.
void trim_idle()
{
    // take the idle contexts off the free list, so that calls on other threads
    // lease fresh contexts instead of waiting while these streams drain
    Ctx* list = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        list = g_free;
        g_free = nullptr;
    }
    if (list == nullptr) { return; }
    Ctx* last = list;
    for (Ctx* c = list; c != nullptr; c = c->next) {
        for (cudaStream_t s : {c->stream, c->side, c->aux}) {
            if (s != nullptr) { cudaStreamSynchronize(s); }
        }
        for (auto& b : c->d) {
            if (b.p != nullptr) { cudaFreeAsync(b.p, c->stream); }
            b.p = nullptr;
            b.cap = 0;
        }
        cudaStreamSynchronize(c->stream);
        for (void* p : c->h_retired) { cudaFreeHost(p); }
        c->h_retired.clear();
        last = c;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    last->next = g_free;
    g_free = list;
    if (g_pool != nullptr) { cudaMemPoolTrimTo(g_pool, 0); }
}

// A context's buffers are used only by its own calls, which have finished
// (or are ordered behind it by call_begin) when the next call reserves, so
// freeing on the context's stream is enough.
bool dreserve(Ctx* c, BufId id, size_t bytes)
{
    DBuf& b = c->d[id];
    if (bytes <= b.cap) { return true; }
    if (b.p != nullptr) {
        cudaFreeAsync(b.p, c->stream);
        b.p = nullptr;
        b.cap = 0;
    }
    size_t want = bytes + bytes / 4 + 4096;
    if (cudaMallocFromPoolAsync(&b.p, want, g_pool, c->stream) != cudaSuccess) {
        // idle contexts keep the buffers of their largest call: give those
        // back and try once more
        cudaGetLastError();
        b.p = nullptr;
        trim_idle();
        if (cudaMallocFromPoolAsync(&b.p, want, g_pool, c->stream) == cudaSuccess) {
            g_allocs.fetch_add(1, std::memory_order_relaxed);
            b.cap = want;
            return true;
        }
        cudaGetLastError();
        b.p = nullptr;
        char msg[128];
        snprintf(msg, sizeof(msg), "device allocation of %zu bytes failed", want);
        tcg_host_set_error(TCG_ERR_OUT_OF_MEMORY, msg);
        return false;
    }
    g_allocs.fetch_add(1, std::memory_order_relaxed);
    b.cap = want;
    return true;
}

bool hreserve(Ctx* c, int id, size_t bytes)
{
    HBuf& b = c->h[id];
    if (bytes <= b.cap) { return true; }
    if (b.p != nullptr) {
        c->h_retired.push_back(b.p);
        b.p = nullptr;
        b.cap = 0;
    }
    // pinning host memory takes tens of milliseconds and holds up other CUDA
    // calls meanwhile, so these small staging buffers grow by doubling from
    // 16 MB and rarely grow at all
    size_t want = std::max<size_t>(bytes * 2u, 16u << 20);
    if (cudaMallocHost(&b.p, want) != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        tcg_host_set_error(TCG_ERR_OUT_OF_MEMORY, "pinned host allocation failed");
        return false;
    }
    g_allocs.fetch_add(1, std::memory_order_relaxed);
    b.cap = want;
    return true;
}

}  // namespace tcg

extern "C" int32_t tcg_init(int32_t device)
{
    std::lock_guard<std::mutex> lk(tcg::g_mu);
    return tcg::init_locked(device) ? 0 : TCG_ERR_INVALID_ARGUMENT;
}

extern "C" void tcg_shutdown(void)
{
    std::lock_guard<std::mutex> lk(tcg::g_mu);
    tcg::Ctx* c = tcg::g_free;
    while (c != nullptr) {
        tcg::Ctx* n = c->next;
        // all of the context's streams are idle before its buffers go
        for (cudaStream_t s : {c->stream, c->side, c->aux}) {
            if (s != nullptr) { cudaStreamSynchronize(s); }
        }
        for (auto& b : c->d) { if (b.p) { cudaFreeAsync(b.p, c->stream); } }
        if (c->stream != nullptr) { cudaStreamSynchronize(c->stream); }
        for (auto& b : c->h) { if (b.p) { cudaFreeHost(b.p); } }
        for (void* p : c->h_retired) { cudaFreeHost(p); }
        for (cudaEvent_t e : {c->fork, c->join, c->afork, c->ajoin, c->gate, c->t0, c->t1}) {
            if (e != nullptr) { cudaEventDestroy(e); }
        }
        for (auto& e : c->kev) { if (e) { cudaEventDestroy(e); } }
        for (cudaStream_t s : {c->stream, c->side, c->aux}) {
            if (s != nullptr) { cudaStreamDestroy(s); }
        }
        delete c;
        c = n;
    }
    tcg::g_free = nullptr;
}

extern "C" uint64_t tcg_launch_count(void)
{
    return tcg::g_launches.load(std::memory_order_relaxed);
}

// Device (cudaMalloc) and pinned host (cudaMallocHost) allocations the library
// has made since it was loaded; a test of an allocation-free call reads it
// before and after.
extern "C" __attribute__((visibility("default"))) uint64_t tcg_allocation_count(void)
{
    return tcg::g_allocs.load(std::memory_order_relaxed);
}

extern "C" double tcg_last_ms(void) { return tcg::t_last_ms; }

extern "C" uint32_t tcg_pipeline_chunks(int32_t decode, const uint64_t* frame_bytes, uint32_t count, uint32_t* starts)
{
    return tcg::pipeline_plan(decode != 0, frame_bytes, count, starts);
}

extern "C" void tcg_prof_enable(int32_t on) { tcg::g_prof_on.store(on != 0 ? 1 : 0); }

extern "C" void tcg_prof_reset(void)
{
    std::lock_guard<std::mutex> lk(tcg::g_mu);
    for (int i = 0; i < tcg::K_COUNT; ++i) { tcg::g_prof_ms[i] = 0.0; tcg::g_prof_n[i] = 0; }
}

extern "C" int32_t tcg_prof_read(uint32_t id, const char** name, double* ms, uint64_t* launches)
{
    if (id >= (uint32_t)tcg::K_COUNT) { return -1; }
    std::lock_guard<std::mutex> lk(tcg::g_mu);
    if (name) { *name = tcg::k_names[id]; }
    if (ms) { *ms = tcg::g_prof_ms[id]; }
    if (launches) { *launches = tcg::g_prof_n[id]; }
    return 0;
}

extern "C" void tcg_set_lease_class(int32_t cls)
{
    tcg::t_lease_class = cls < 0 ? -1 : cls;
}

extern "C" void tcg_trim_idle(void)
{
    if (tcg::ensure_init()) { tcg::trim_idle(); }
}

extern "C" int32_t tcg_pool_reserve(uint64_t bytes)
{
    if (!tcg::ensure_init()) { return TCG_ERR_NOT_IMPLEMENTED; }
    if (bytes == 0u) { return 0; }
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return TCG_ERR_OUT_OF_MEMORY;
    }
    void* p = nullptr;
    int32_t rc = 0;
    if (cudaMallocFromPoolAsync(&p, bytes, tcg::g_pool, s) == cudaSuccess) {
        cudaFreeAsync(p, s);
    } else {
        cudaGetLastError();
        rc = TCG_ERR_OUT_OF_MEMORY;
    }
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}

// Free device memory as the library can use it: the device's free memory plus
// what the library's pool holds mapped but unused.
extern "C" void tcg_mem_info(uint64_t* free_bytes, uint64_t* total_bytes)
{
    size_t f = 0, t = 0;
    if (!tcg::ensure_init() || cudaMemGetInfo(&f, &t) != cudaSuccess) {
        cudaGetLastError();
        f = t = 0;
    }
    uint64_t reserved = 0, used = 0;
    if (f != 0u && tcg::g_pool != nullptr &&
        cudaMemPoolGetAttribute(tcg::g_pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(tcg::g_pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
        reserved > used) {
        f += reserved - used;
    }
    cudaGetLastError();
    *free_bytes = f;
    *total_bytes = t;
}

extern "C" int32_t tcg_is_device_ptr(const void* p)
{
    if (p == nullptr) { return 0; }
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

extern "C" int32_t tcg_read_device(void* dst, const void* src, size_t n)
{
    if (n == 0u) { return 0; }
    if (!tcg::ensure_init()) { return TCG_ERR_NOT_IMPLEMENTED; }
    TCG_CHECK(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost));
    return 0;
}
