/* topos_codec.h - public C ABI of the B200 Topos Codec intra frame library.
 *
 * This header declares the drop-in subset of the Topos Codec C ABI that the
 * GPU library implements, with struct layouts identical to the reference ABI
 * version 2 (reference: native/include/topos_codec.h). Every declaration cites
 * the reference declaration it replaces. Callers built against the reference
 * header can link against this library unchanged for the frame path.
 *
 * Conventions (same as the reference ABI):
 *  - Every public struct starts with struct_size then abi_version. Callers
 *    zero-initialise; 0 in either field means "current". The library writes
 *    struct_size = sizeof on structs it fills.
 *  - Status codes are frozen; negative = error, TC_WARN_CONCEALED = +1.
 *  - Returned const char* strings are library-owned (static or thread-local).
 *  - All frame functions are re-entrant: state is caller-owned, errors are
 *    thread-local, device work is issued on per-call stream leases.
 *
 * The tcg_* functions at the end are extensions that do not exist in the
 * reference ABI (batched encode, device-resident buffers, serving loop); they
 * change no reference symbol's behaviour.
 */
#ifndef TOPOS_CODEC_H
#define TOPOS_CODEC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* reference: native/include/topos_codec.h:31 */
#define TOPOS_CODEC_ABI_VERSION 2

/* Status codes. reference: native/include/topos_codec.h:34-56 */
enum {
    TC_OK                           =   0,
    TC_WARN_CONCEALED               =   1,
    TC_ERR_INVALID_ARGUMENT         =  -1,
    TC_ERR_OUT_OF_MEMORY            =  -2,
    TC_ERR_UNSUPPORTED_VERSION      =  -3,
    TC_ERR_UNSUPPORTED_PROFILE      =  -4,
    TC_ERR_UNSUPPORTED_PIXEL_FORMAT =  -5,
    TC_ERR_UNSUPPORTED_MATRIX       =  -6,
    TC_ERR_UNSUPPORTED_ALPHA_MODE   =  -7,
    TC_ERR_LIMIT_EXCEEDED           =  -8,
    TC_ERR_MALFORMED                =  -9,
    TC_ERR_TRUNCATED                = -10,
    TC_ERR_CHECKSUM_MISMATCH        = -11,
    TC_ERR_STATE                    = -12,
    TC_ERR_CANCELLED                = -13,
    TC_ERR_IO                       = -14,
    TC_ERR_BUFFER_TOO_SMALL         = -15,
    TC_ERR_NOT_IMPLEMENTED          = -16,
    TC_ERR_REFERENCE_INVALID        = -17
};

/* reference: native/include/topos_codec.h:58-67 */
typedef struct topos_version_info {
    uint32_t    struct_size;
    uint32_t    abi_version;
    uint32_t    version_major;
    uint32_t    version_minor;
    uint32_t    version_patch;
    const char* git_commit;
    const char* build_target;
    uint32_t    reserved[4];
} topos_version_info;

/* reference: native/include/topos_codec.h:70-80 */
#define TOPOS_CPU_X86_AVX2    (1u << 0)
#define TOPOS_CPU_X86_AVX512F (1u << 1)
#define TOPOS_CPU_ARM_NEON    (1u << 2)
#define TOPOS_CPU_X86_FMA     (1u << 3)

typedef struct topos_cpu_features {
    uint32_t struct_size;
    uint32_t abi_version;
    uint32_t flags;
    uint32_t reserved[5];
} topos_cpu_features;

/* reference: native/include/topos_codec.h:84-104 */
#define TC_CODEC_CAP_FULL_DECODE               (1u << 0)
#define TC_CODEC_CAP_FIXED_REDUCED_DECODE      (1u << 1)
#define TC_CODEC_CAP_AUTO_2K_DECODE            (1u << 2)
#define TC_CODEC_CAP_CPU_SURFACE_OUTPUT        (1u << 3)
#define TC_CODEC_CAP_HOST_VISIBLE_GPU_SURFACE  (1u << 4)
#define TC_CODEC_CAP_V7A_BAND_DECODE           (1u << 5)
#define TC_CODEC_CAP_V7B_SCALABLE_BASE         (1u << 6)
#define TC_CODEC_CAP_DECODE_DROP_ALPHA         (1u << 7)

#define TC_CODEC_MAX_DIM 16384u
#define TC_CODEC_AUTO_2K_MAX_DIM 2048u

typedef struct topos_codec_capabilities {
    uint32_t struct_size;
    uint32_t abi_version;
    uint32_t flags;
    uint32_t max_width;
    uint32_t max_height;
    uint32_t auto2k_max_dim;
    uint32_t reserved[4];
} topos_codec_capabilities;

/* reference: native/include/topos_codec.h:125 */
int32_t tc_abi_version(void);
/* reference: native/include/topos_codec.h:128 */
int32_t tc_version(topos_version_info* out);
/* reference: native/include/topos_codec.h:131 */
int32_t tc_query_cpu_features(topos_cpu_features* out);
/* reference: native/include/topos_codec.h:135. This library advertises
 * FULL_DECODE | CPU_SURFACE_OUTPUT (the paths it implements). */
int32_t tc_query_capabilities(topos_codec_capabilities* out);
/* reference: native/include/topos_codec.h:142 */
int32_t tc_query_support(uint32_t profile, uint32_t pixel_format, uint32_t bit_depth,
                         uint32_t alpha_mode);
/* reference: native/include/topos_codec.h:146 */
const char* tc_status_message(int32_t status);
/* reference: native/include/topos_codec.h:150 */
const char* tc_last_error(void);

/* ============================ frame coding ============================ */

/* reference: native/include/topos_codec.h:168-173 */
#define TC_FRAME_MAX_PLANES 4
#define TC_FRAME_DEFAULT_SLICE_ROWS 16u

/* reference: native/include/topos_codec.h:177-224. reserved[0] low byte selects
 * the coding generation; this library encodes 8 (V7-R2 rANS2 intra) and
 * reserved[5] carries the V7-R2 output features (bit0 DEBLOCK, bit1 QPT2). */
typedef struct topos_frame_config {
    uint32_t struct_size;
    uint32_t abi_version;
    uint16_t visible_width;
    uint16_t visible_height;
    uint8_t profile;
    uint8_t pixel_format;     /* 0 YUV 4:2:2, 1 YUV 4:4:4, 2 GBR, 3 CFA */
    uint8_t bit_depth;
    uint8_t qmatrix_id;
    uint8_t qp_base;
    int8_t qp_delta_luma;
    int8_t qp_delta_chroma;
    uint8_t slice_rows;       /* block rows per slice; 0 = 16 */
    uint8_t alpha_mode;       /* 0 none, 1 lossless, 2 near-lossless */
    uint8_t alpha_bit_depth;
    uint8_t alpha_premultiplied;
    uint8_t color_range;
    uint8_t color_primaries;
    uint8_t color_transfer;
    uint8_t color_matrix;
    uint8_t chroma_siting;
    uint16_t sar_num;
    uint16_t sar_den;
    uint32_t reserved[8];
} topos_frame_config;

/* reference: native/include/topos_codec.h:231-237. Strides are in uint16
 * elements; 0 = tight. */
typedef struct topos_frame_input {
    uint32_t struct_size;
    uint32_t abi_version;
    const uint16_t* planes[TC_FRAME_MAX_PLANES];
    size_t strides[TC_FRAME_MAX_PLANES];
    uint32_t reserved[8];
} topos_frame_input;

/* reference: native/include/topos_codec.h:240-254 */
typedef struct topos_frame_stats {
    uint32_t struct_size;
    uint32_t abi_version;
    uint32_t packet_size;
    uint32_t color_payload_bytes;
    uint32_t alpha_payload_bytes;
    uint32_t color_header_bytes;
    uint32_t alpha_header_bytes;
    uint16_t slice_count;
    uint8_t qp_base;
    uint8_t reserved8;
    uint16_t alpha_max_abs_error;
    uint16_t reserved16;
    uint32_t reserved[8];
} topos_frame_stats;

/* reference: native/include/topos_codec.h:257-285 */
#define TC_FRAME_SLICE_OK 0u
#define TC_FRAME_SLICE_CONCEALED 1u
#define TC_MAX_SLICES 512

typedef struct topos_frame_output {
    uint32_t struct_size;
    uint32_t abi_version;
    uint16_t visible_width;
    uint16_t visible_height;
    uint16_t coded_width;
    uint16_t coded_height;
    uint8_t plane_count;
    uint8_t bit_depth;
    uint8_t profile;
    uint8_t pixel_format;
    uint8_t alpha_mode;
    uint8_t alpha_bit_depth;
    uint8_t color_range;
    uint8_t color_primaries;
    uint8_t color_transfer;
    uint8_t color_matrix;
    uint8_t chroma_siting;
    uint16_t concealed_slices;
    uint16_t slice_count;
    uint16_t sar_num;
    uint16_t sar_den;
    uint8_t slice_status[TC_MAX_SLICES];
    uint32_t reserved[8];
} topos_frame_output;

/* reference: native/include/topos_codec.h:288 (rules: native/src/codec/codec.c:426-605) */
int32_t tc_frame_config_validate(const topos_frame_config* cfg);

/* reference: native/include/topos_codec.h:292 (native/src/codec/codec.c:607-647) */
size_t tc_frame_packet_bound(const topos_frame_config* cfg);

/* reference: native/include/topos_codec.h:296 (native/src/codec/codec.c:5970-6018).
 * Fixed-QP V7-R2 encode on the GPU. out is written only on success;
 * out == NULL with out_cap == 0 is a size probe (BUFFER_TOO_SMALL + stats). */
int32_t tc_frame_encode(const topos_frame_config* cfg, const topos_frame_input* input,
                        uint8_t* out, size_t out_cap, topos_frame_stats* stats);

/* reference: native/include/topos_codec.h:336 (native/src/codec/codec.c:9005-9098).
 * planes_out == NULL = query mode (geometry only). Damaged slices are
 * concealed and the call returns TC_WARN_CONCEALED. */
int32_t tc_frame_decode(const uint8_t* data, size_t size,
                        uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                        const size_t strides[TC_FRAME_MAX_PLANES],
                        topos_frame_output* out_info);

/* reference: native/include/topos_codec.h:387-390 */
typedef struct topos_batch_packet {
    const uint8_t* data;
    size_t size;
} topos_batch_packet;

/* reference: native/include/topos_codec.h:398 (native/src/codec/codec.c:9639-9805).
 * planes_out is count x TC_FRAME_MAX_PLANES (row = frame); strides same shape
 * or NULL. All frames' slices are decoded in one device launch sequence. */
int32_t tc_frame_decode_batch(const topos_batch_packet* packets, uint32_t count,
                              uint16_t* const* planes_out, const size_t* strides,
                              topos_frame_output* infos);

/* reference: native/include/topos_codec.h:410 (native/src/codec/codec.c:9807-9831) */
int32_t tc_frame_plane_geometry(const topos_frame_output* info, uint32_t plane,
                                uint32_t* width, uint32_t* height);

/* ==================== extensions (no reference counterpart) ==================== */

/* Batched encode: count frames (any mix of geometries and configs) coded in one
 * device launch sequence. outs[i]/out_caps[i] receive frame i's packet; stats[i]
 * (array of count, may be NULL) receives its stats; rcs[i] its status. Returns
 * the first non-OK frame status (frame order), TC_OK otherwise. Each frame's
 * packet is byte-identical to tc_frame_encode of that frame alone. */
int32_t tcg_frame_encode_batch(const topos_frame_config* cfgs,
                               const topos_frame_input* inputs, uint32_t count,
                               uint8_t* const* outs, const size_t* out_caps,
                               topos_frame_stats* stats, int32_t* rcs);

/* Allocation-free packet query. No counterpart in the reference: it exists for
 * callers that must not allocate device memory while they run - a serving
 * process whose GPU memory is handed out up front by its own pool (a stray
 * cudaMalloc can fail there once the pool holds the free memory, and it breaks
 * the pool's accounting), and latency-critical threads, because cudaMalloc and
 * cudaFree may synchronise the whole device and stall the work of others.
 *
 * Returns, for count packets, the same frame information (and the same status)
 * as tc_frame_decode_batch(packets, count, NULL, NULL, infos). Packets may sit
 * in device memory (their headers are walked on the GPU) or in host memory.
 * The call allocates nothing, in device or host memory: its device scratch
 * (~550 KB) is a static array of the library that every GPU loading the
 * library holds until the process exits. Limits and rules:
 *  - at most TCG_NOALLOC_MAX_PACKETS packets per call; more is rejected with
 *    TC_ERR_LIMIT_EXCEEDED before any device work;
 *  - the first call on a device looks up the scratch address on that device
 *    (which may load the library's device code there); make that first call
 *    before any CUDA stream capture is in progress;
 *  - the scratch is shared by every call on a device and keeps the last call's
 *    records; each call clears the records it uses before writing them, but
 *    calls that overlap on the GPU (from several host threads at once) race on
 *    it, so serialise them;
 *  - the call runs on the default stream of the calling thread's current
 *    device and returns when its device work has finished; a packet in the
 *    memory of another device is rejected with TC_ERR_INVALID_ARGUMENT (make
 *    the packets' device current first). */
#define TCG_NOALLOC_MAX_PACKETS 64u
int32_t tcg_frame_query_batch_noalloc(const topos_batch_packet* packets, uint32_t count,
                                      topos_frame_output* infos);

/* Batched V8 decode. No counterpart in the reference, whose
 * tc_frame_decode_batch takes V7 packets only: count V8 packets (host or
 * device memory) decoded in one device launch sequence, each frame with the
 * result tc_frame_decode gives it (planes, per-tile slice_status,
 * concealed_slices). Every packet is scanned and checked before any decode;
 * a failing packet fails the call with its status. planes_out (count x 4) NULL
 * = query only; strides (count x 4) NULL = tight rows. */
int32_t tcg_frame_decode_v8_batch(const topos_batch_packet* packets, uint32_t count, uint16_t* const* planes_out,
                                  const size_t* strides, topos_frame_output* infos);

/* Continuous-batching request server (no counterpart in the reference).
 * Encode and decode requests of single frames (any mix of sizes,
 * configurations and generations, V7-R2 or V8; buffers owned by the caller,
 * host or device memory, valid until the request completes) enter two
 * queues. Each direction has a pool of workers, each on its own CUDA stream:
 * an idle worker codes the requests that have arrived (an even share when
 * other workers are idle too, at most max_batch_frames, 1..64) in one batched
 * call, and requests arriving while batches run are taken by the next idle
 * worker at once, so their work overlaps the batches already on the GPU.
 * Half of each direction's workers (rounded down) take frames up to
 * 2560x1440 only. A batch admits requests while the estimated device bytes
 * of all batches in flight fit max_bytes_in_flight (0 = no limit) and 7/8 of
 * the device memory that was free when the server was created (it is read
 * once: querying it while requests run stalled them). A worker that finds
 * fewer than four V7-R2 requests waits up to 4 ms for more; V8 requests go at
 * once. Creating a server maps up to half of the free device
 * memory (at most 64 GB) into the library's memory pool, so that workers'
 * buffers do not map memory while other requests run; tcg_release_idle_memory
 * gives back what idle contexts hold.
 * Every result equals the single-frame call's. tcg_server_wait blocks until
 * the ticket's request is done and returns its status (as tc_frame_encode /
 * tc_frame_decode would), its stats or frame information, and its latency
 * from submission to completion. Decode requests are validated on
 * submission: an invalid packet returns its error there.
 * tcg_server_create uses 4 workers per direction; tcg_server_create_ex takes
 * the count (1..16). */
typedef struct tcg_server tcg_server;
int32_t tcg_server_create(uint64_t max_bytes_in_flight, uint32_t max_batch_frames, tcg_server** out);
int32_t tcg_server_create_ex(uint64_t max_bytes_in_flight, uint32_t max_batch_frames, uint32_t workers,
                             tcg_server** out);
void tcg_server_destroy(tcg_server* server);
int32_t tcg_server_submit_encode(tcg_server* server, const topos_frame_config* cfg, const topos_frame_input* input,
                                 uint8_t* out, size_t out_cap, uint64_t* ticket);
int32_t tcg_server_submit_decode(tcg_server* server, const uint8_t* packet, size_t size,
                                 uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                                 const size_t strides[TC_FRAME_MAX_PLANES], uint64_t* ticket);
int32_t tcg_server_wait(tcg_server* server, uint64_t ticket, int32_t* status, topos_frame_stats* stats,
                        topos_frame_output* info, double* latency_ms);

/* ---------------- decode delivery modes and persistent decoder contexts ----------------
 * Reference: native/include/topos_codec.h:340-380 (scaled and reduced decode),
 * :425-572 (plane views, requests, surfaces, decoder contexts); behaviour
 * native/src/codec/codec.c:9100-9376 and 9378-9805, decoder_ctx.c. Types and
 * layouts are the reference's. A decode request selects the delivered grid:
 * FULL (source size), SCALED (target_width x target_height, each target
 * sample the reconstruction at (x * source / target) rounded down), REDUCED
 * (fixed ratio 1/2, 1/3, 1/4, 1/8: the same sampling of a reconstruction
 * that keeps the first 24, 16, 10 or 4 zigzag coefficients) or AUTO_2K (the
 * source when it fits 2048x2048, else the first reduced ratio that does,
 * or an explicit target). Deblocking runs on the delivered planes: on the
 * 8-sample grid at full size, on the 4-sample grid for an exact half, not at
 * all for other scaled grids. DROP_ALPHA skips the alpha slices (reported
 * OK, unchecked) and delivers three planes. Every pointer may be host or
 * device memory. Decoder contexts hold no state the result depends on: they
 * are thin handles over the stateless calls. */
typedef enum tc_decode_scale {
    TC_DECODE_SCALE_FULL = 0,
    TC_DECODE_SCALE_HALF = 1,
    TC_DECODE_SCALE_THIRD = 2,
    TC_DECODE_SCALE_QUARTER = 3,
    TC_DECODE_SCALE_EIGHTH = 4
} tc_decode_scale;

typedef struct topos_plane_view {
    uint32_t struct_size;
    uint32_t abi_version;
    uint16_t* pixels;
    size_t stride;          /* uint16 elements; 0 = tight */
} topos_plane_view;

enum {
    TC_DECODE_MEMORY_CPU = 0u,
    TC_DECODE_MEMORY_HOST_VISIBLE_GPU = 1u
};

typedef enum topos_decode_mode {
    TC_DECODE_MODE_FULL = 0u,
    TC_DECODE_MODE_SCALED = 1u,
    TC_DECODE_MODE_REDUCED = 2u,
    TC_DECODE_MODE_AUTO_2K = 3u
} topos_decode_mode;

typedef enum tc_decode_quality {
    TC_DECODE_QUALITY_DEFAULT = 0u,
    TC_DECODE_QUALITY_FAST = 1u,
    TC_DECODE_QUALITY_BALANCED = 2u,
    TC_DECODE_QUALITY_HIGH = 3u
} tc_decode_quality;

typedef struct topos_decode_request {
    uint32_t struct_size;
    uint32_t abi_version;
    uint32_t mode;          /* topos_decode_mode */
    uint32_t scale;         /* tc_decode_scale; REDUCED only */
    uint32_t target_width;  /* SCALED / AUTO_2K; 0 together with height */
    uint32_t target_height;
    uint32_t quality;       /* tc_decode_quality; checked and kept */
    uint32_t memory_type;   /* TC_DECODE_MEMORY_* */
    uint32_t flags;         /* TC_DECODE_FLAG_* */
    uint32_t reserved[4];   /* zero */
} topos_decode_request;

#define TC_DECODE_FLAG_DROP_ALPHA (1u << 0)

typedef struct topos_decode_surface {
    uint32_t struct_size;
    uint32_t abi_version;
    uint32_t memory_type;
    uint32_t reserved;
    topos_plane_view planes[TC_FRAME_MAX_PLANES];
} topos_decode_surface;

typedef struct topos_decoder_config {
    uint32_t struct_size;
    uint32_t abi_version;
    uint32_t max_slice_workers; /* kept; the GPU decode has no host worker pool */
    uint32_t reserved[7];
} topos_decoder_config;

typedef struct tc_decoder tc_decoder;

/* ceil(source / 1, 2, 3, 4, 8) */
int32_t tc_decode_scale_dimensions(uint32_t source_width, uint32_t source_height, tc_decode_scale scale,
                                   uint32_t* target_width, uint32_t* target_height);
int32_t tc_frame_decode_scaled(const uint8_t* data, size_t size, uint32_t target_width, uint32_t target_height,
                               uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                               const size_t strides[TC_FRAME_MAX_PLANES], topos_frame_output* out_info);
int32_t tc_frame_decode_reduced(const uint8_t* data, size_t size, tc_decode_scale scale,
                                uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                                const size_t strides[TC_FRAME_MAX_PLANES], topos_frame_output* out_info);
int32_t tc_frame_decode_batch_reduced(const topos_batch_packet* packets, uint32_t count, tc_decode_scale scale,
                                      uint16_t* const* planes_out, const size_t* strides, topos_frame_output* infos);
int32_t tc_frame_decode_request(const uint8_t* data, size_t size, const topos_decode_request* request,
                                uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                                const size_t strides[TC_FRAME_MAX_PLANES], topos_frame_output* out_info);

int32_t tc_decoder_create(const topos_decoder_config* cfg, tc_decoder** out);
void tc_decoder_destroy(tc_decoder* dec);
int32_t tc_decoder_set_max_slice_workers(tc_decoder* dec, uint32_t workers);
int32_t tc_decoder_prepare(tc_decoder* dec, const uint8_t* packet, size_t size, topos_frame_output* info);
int32_t tc_decoder_prepare_request(tc_decoder* dec, const uint8_t* packet, size_t size,
                                   const topos_decode_request* request, topos_frame_output* info);
int32_t tc_decoder_decode(tc_decoder* dec, const uint8_t* packet, size_t size,
                          const topos_plane_view out[TC_FRAME_MAX_PLANES], topos_frame_output* info);
int32_t tc_decoder_decode_request(tc_decoder* dec, const uint8_t* packet, size_t size,
                                  const topos_decode_request* request,
                                  const topos_plane_view out[TC_FRAME_MAX_PLANES], topos_frame_output* info);
int32_t tc_decoder_decode_batch(tc_decoder* dec, const topos_batch_packet* packets, uint32_t count,
                                const topos_plane_view* out, topos_frame_output* infos);
int32_t tc_decoder_decode_batch_request(tc_decoder* dec, const topos_batch_packet* packets, uint32_t count,
                                        const topos_decode_request* request, const topos_plane_view* out,
                                        topos_frame_output* infos);
int32_t tc_decoder_decode_surface(tc_decoder* dec, const uint8_t* packet, size_t size,
                                  const topos_decode_surface* surface, topos_frame_output* info);
int32_t tc_decoder_decode_surface_request(tc_decoder* dec, const uint8_t* packet, size_t size,
                                          const topos_decode_request* request, const topos_decode_surface* surface,
                                          topos_frame_output* info);

/* ---------------- MOV read path and its hand-off to the batched decoder ----------------
 * Reference: native/include/topos_codec.h:655-770 (io, movie information) and
 * 880-1014 (reader calls); behaviour native/src/mov/mov.c:2260-2760 (atoms and
 * sample tables), 3642-4182 (open, information), 4419-4770 (packets, timing,
 * sync). The video track of a QuickTime file written by the reference muxer:
 * open indexes the sample table without reading samples; packet and batch
 * reads check every packet's header against the track's tpcC configuration.
 * Audio and timecode tracks are skipped unparsed. tcg_movie_decode_batch
 * (extension) reads samples [start, start + count) with one read when they lie
 * back to back and decodes them as one tc_frame_decode_batch. */
typedef int32_t (*tc_io_read_fn)(void* ctx, uint64_t offset, void* buf, size_t len);
typedef int32_t (*tc_io_write_fn)(void* ctx, const void* data, size_t len);
typedef int32_t (*tc_io_seek_write_fn)(void* ctx, uint64_t offset, const void* data, size_t len);

typedef struct topos_io {
    uint32_t struct_size;
    uint32_t abi_version;
    void* ctx;
    tc_io_read_fn read;
    tc_io_write_fn write;
    tc_io_seek_write_fn seek_write;
    uint64_t length;           /* reader: bytes of the source */
    uint32_t reserved[4];
} topos_io;

#define TC_MOVIE_MAX_SAMPLES 67108864u

typedef struct topos_movie_info {
    uint32_t struct_size;
    uint32_t abi_version;
    uint16_t visible_width;
    uint16_t visible_height;
    uint8_t profile;
    uint8_t pixel_format;
    uint8_t bit_depth;
    uint8_t qmatrix_id;
    uint8_t qp_base;
    int8_t qp_delta_luma;
    int8_t qp_delta_chroma;
    uint8_t alpha_mode;
    uint8_t alpha_bit_depth;
    uint8_t alpha_premultiplied;
    uint8_t color_range;
    uint8_t color_primaries;
    uint8_t color_transfer;
    uint8_t color_matrix;
    uint8_t chroma_siting;
    uint16_t sar_num;
    uint16_t sar_den;
    uint32_t timescale;
    uint32_t sample_count;
    uint32_t faststart;        /* 1 = moov before mdat */
    uint32_t index_bytes;
    uint32_t reserved[8];      /* [0] tpcC bitstream major, [1] tpcD tier */
} topos_movie_info;

typedef struct topos_alpha_budget_info {
    uint32_t struct_size;
    uint32_t abi_version;
    uint16_t target_ratio_bp;
    uint16_t actual_ratio_bp;
    uint16_t max_abs_error;
    uint16_t flags;
    uint32_t frame_count;
    uint32_t reserved[4];
} topos_alpha_budget_info;

typedef struct topos_movie topos_movie;

int32_t tc_movie_open(const topos_io* io, topos_movie** out);
int32_t tc_movie_open_fd(int fd, uint64_t length, topos_movie** out);
int32_t tc_movie_info(const topos_movie* movie, topos_movie_info* info);
int32_t tc_movie_alpha_budget(const topos_movie* movie, topos_alpha_budget_info* info);
int32_t tc_movie_packet(const topos_movie* movie, uint32_t sample_index, uint8_t* buf, size_t cap, size_t* need_size);
int32_t tc_movie_packet_base(const topos_movie* movie, uint32_t sample_index, uint8_t* buf, size_t cap,
                             size_t* need_size);
int32_t tc_movie_packet_batch(const topos_movie* movie, uint32_t start, uint32_t count, uint8_t* arena, size_t cap,
                              size_t* offsets_out, size_t* sizes_out, size_t* need_total);
int32_t tc_movie_packet_base_batch(const topos_movie* movie, uint32_t start, uint32_t count, uint8_t* arena,
                                   size_t cap, size_t* offsets_out, size_t* sizes_out, uint8_t* base_flags_out,
                                   size_t* need_total);
int32_t tc_movie_packet_pts(const topos_movie* movie, uint32_t sample_index, uint64_t* pts_tick, uint32_t* dur_tick);
int32_t tc_movie_packet_sync(const topos_movie* movie, uint32_t sample_index, uint8_t* is_sync);
int32_t tc_movie_prev_sync(const topos_movie* movie, uint32_t sample_index, uint32_t* sync_index);
void tc_movie_close(topos_movie* movie);

/* Decodes movie samples [start, start + count) as one batch: planes_out,
 * strides and infos as in tc_frame_decode_batch (planes_out NULL = frame
 * information only). Returns the first failing status of the sample reads
 * (no frame decoded) or of the decode. */
int32_t tcg_movie_decode_batch(const topos_movie* movie, uint32_t start, uint32_t count, uint16_t* const* planes_out,
                               const size_t* strides, topos_frame_output* infos);

/* Decode-chain tiling chosen for batches of the given number of colour slices:
 * one lane per slice with 8 (0), 4 (2), 2 (3) or 1 (4) slices per warp, one
 * warp per slice (1), or a split (5: the largest slices, half of the blocks,
 * one per warp and the rest four per warp on a second stream); -1 = not
 * chosen yet. The first batch of each size class (log2 of the slice count)
 * times the split and 4, 2 and 1 slices per warp and keeps the fastest;
 * the environment variable TCG_DCHAIN=lane|lane4|lane2|lane1|warp|split overrides
 * the choice ("lane" is 8 per warp). All produce identical output. */
int32_t tcg_dchain_tiling(uint32_t colour_slices);

/* Size-targeted encode of many frames (extension beside tc_frame_encode_sized):
 * frame i is searched for target_bytes[i] in [qp_min, qp_max] exactly as a
 * tc_frame_encode_sized call made while another call holds the cross-call qp
 * hint (an empty hint record), so the results do not depend on frame order.
 * Up to six searches run side by side on their own contexts (fewer when
 * their probe windows would take more than 96 GB of device memory), so their
 * probe launches overlap on the GPU. Per frame: rcs[i] (as the single call
 * returns), qp_used[i] (may be NULL), stats[i] (may be NULL) and the packet in
 * outs[i] (NULL = size only, capacity out_caps[i]). Returns the first nonzero
 * rcs[i], or TC_OK. tc_last_error describes only errors of argument checks
 * made on the calling thread. */
int32_t tcg_frame_encode_sized_batch(const topos_frame_config* cfgs, const topos_frame_input* inputs, uint32_t count,
                                     const uint32_t* target_bytes, uint8_t qp_min, uint8_t qp_max, uint8_t* qp_used,
                                     uint8_t* const* outs, const size_t* out_caps, topos_frame_stats* stats,
                                     int32_t* rcs);

/* Batches whose inputs or outputs are in host memory are coded as chunks on
 * separate streams (encode up to four, decode up to three): chunk i's
 * host-to-device copies queue behind chunk i-1's, so the copies of later
 * chunks overlap the kernels of earlier ones and each chunk's results return
 * while later chunks still compute. A batch is chunked when its host copy
 * bytes (encode: samples; decode: packets plus planes) reach 256 MB, one chunk
 * per 64 MB. The output is identical to the unchunked call's.
 * tcg_pipeline_plan reports the split the library would use for an encode
 * (decode = 0) or decode (decode != 0) batch with the given per-frame copy
 * bytes: it returns the chunk count k (1 = no chunking) and fills starts[0..k]
 * (frames [starts[i], starts[i+1]) form chunk i; starts must hold 5 entries).
 * The environment variable TCG_PIPELINE=<n> forces n chunks (0 or 1: never
 * chunk; at most four). Host work only; needs no device. */
uint32_t tcg_pipeline_plan(int32_t decode, const uint64_t* frame_bytes, uint32_t count, uint32_t* starts);

/* Device selection and teardown for the calling process. tcg_device_init is
 * implicit on first use (device 0 or the current CUDA device). */
int32_t tcg_device_init(int32_t device);
void tcg_device_release(void);

/* Give back the device memory of every call context that is not in use.
 * Contexts keep the buffers of their largest call so that the next call of
 * that size allocates nothing; a process that shares the device with another
 * allocator (a framework's caching allocator) calls this between phases. The
 * next call on such a context allocates again. */
void tcg_release_idle_memory(void);

/* Number of device kernel launches issued by this library in this process
 * (diagnostics for benchmarks). */
uint64_t tcg_kernel_launches(void);

/* Device time in milliseconds of the calling thread's last frame call,
 * measured with CUDA events on the stream the call's kernels ran on (from the
 * first upload to the last download; for a chunked host-memory batch, from
 * the first chunk's start to the last chunk's end). */
double tcg_last_device_ms(void);

/* Optional per-kernel timing: when enabled, every kernel launch is bracketed
 * by CUDA events and the durations are summed per kernel for the process.
 * tcg_profile_read(id) returns TC_OK with the kernel's name, total ms and
 * launch count, or a negative value past the last kernel id. */
void tcg_profile_enable(int32_t on);
void tcg_profile_reset(void);
int32_t tcg_profile_read(uint32_t id, const char** name, double* total_ms, uint64_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* TOPOS_CODEC_H */
