/* tc_internal.h - host-side internals of the B200 Topos Codec library (C11).
 *
 * The host library owns everything that is not per-pixel or per-symbol work:
 * configuration and bitstream-header rules, slice planning, packet structure
 * parsing, error semantics and the public entry points. Device work goes
 * through the internal C ABI in tcg_device.h.
 */
#ifndef TC_INTERNAL_H
#define TC_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "../../../include/topos_codec.h"

#define TC_EXPORT __attribute__((visibility("default")))

#define TC_HDR_SIZE 53u
#define TC_SH_SIZE 17u
#define TC_MAX_DIM 16384u
#define TC_MAX_SLICE_COUNT 512u
#define TC_MAX_PACKET 268435456u
#define TC_QP_MAX 95u
#define TC_QP_V15_MIN 64u
#define TC_TRAW_LOG0 20u
#define TC_BATCH_MAX_FRAMES 65536u

/* Frame header fields (53-byte layout of reference
 * native/src/bitstream/frame_header.h:28-70) plus derived plane geometry. */
typedef struct tc_hdr {
    uint8_t major, minor;
    uint16_t flags;
    uint8_t profile, pf, bd, amode, abd, ftype;
    uint16_t gop;
    uint8_t refd;
    uint16_t cw, ch, vw, vh;
    uint8_t planes, qm, qp;
    uint16_t slices;
    uint8_t range, prim, xfer, matrix, siting;
    uint16_t sarn, sard;
    uint32_t size;
    uint8_t em, cb, cm;
    uint16_t pcw[4], pch[4], pvw[4], pvh[4], bcols[4], brows[4];
} tc_hdr;

/* 17-byte slice header (reference native/src/bitstream/slice_map.h:12-23) */
typedef struct tc_shdr {
    uint32_t size;
    uint8_t plane;
    uint16_t y0, bh;
    uint8_t qdb, k1, k2, k3;
    uint32_t crc;
} tc_shdr;

typedef struct tc_view {
    tc_hdr h;
    tc_shdr s[TC_MAX_SLICE_COUNT];
    uint32_t off[TC_MAX_SLICE_COUNT]; /* payload offset within the packet */
} tc_view;

int32_t tc_hdr_decode(const uint8_t* d, size_t n, tc_hdr* h);

/* version_major of a packet in host or device memory (-1: no TPIC header) */
int tc_packet_major(const uint8_t* data, size_t size);

/* ---- V8 segmented rANS packets (tc_v8.c) ---- */
/* single-frame decode or query (planes_out NULL) of a V8 packet, host or device memory */
int32_t tc_v8_frame_decode(const uint8_t* data, size_t size, uint16_t* const planes_out[4], const size_t strides[4],
                           topos_frame_output* o);

/* ---- errors (tc_error.c) ---- */
int32_t tc_fail(int32_t status, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

/* ---- CRC-32 (tc_crc32.c) ---- */
uint32_t tc_crc32(const uint8_t* data, size_t n);

/* ---- tables (tc_tables.c) ---- */
extern const uint8_t tc_zigzag[64];
uint32_t tc_qp_scale(uint32_t refined, uint32_t qp);
/* qmatrix_id -> natural-order table (0 = luma, 1 = chroma); 0 if unknown */
int tc_qmatrix(uint8_t id, int chroma, uint16_t out[64]);
/* Q = max(1, (qm*scale + 128) >> 8) for all 64 positions */
void tc_quant_steps(const uint16_t qm[64], uint32_t qp, uint32_t refined, uint32_t Q[64]);
int64_t tc_coef_clamp(uint8_t bit_depth);
/* exact IEEE-754 log2 series for the model choice (4096 entries, index = freq) */
const double* tc_log2_table(void);

/* ---- header rules (tc_header.c) ---- */
int32_t tc_hdr_validate(const tc_hdr* h);
int32_t tc_hdr_geometry(tc_hdr* h);
void tc_hdr_pack(const tc_hdr* h, uint8_t out[TC_HDR_SIZE]);
void tc_cfg_to_hdr(const topos_frame_config* c, tc_hdr* h);
uint32_t tc_cfg_slice_rows(const topos_frame_config* c);
int32_t tc_band_plan(const tc_hdr* h, uint32_t rows_per, uint32_t* total);
/* generation probe ahead of the structural parse; 0 = continue */
int32_t tc_probe_generation(const uint8_t* d, size_t n);
int32_t tc_parse_structure(const uint8_t* d, size_t n, tc_view* v);
/* same checks from a device walk record (tcg_device.h TCG_WALK_REC layout) */
int32_t tc_parse_compact(const uint8_t* rec, size_t n, tc_view* v);
void tc_fill_info(const tc_hdr* h, topos_frame_output* o);

/* Delivered grid of a decoded frame (reference codec.c:8560-8640, 8700-8745):
 * full size, or scaled to tw x th (4:2:2 chroma ceil(tw/2)) from a
 * reconstruction keeping zigzag positions <= climit; drop_alpha delivers
 * three planes and leaves the alpha slices undecoded. A nonzero tw also
 * reports tw x th as both the visible and the coded size of the frame, as a
 * resolved request does even at full size. */
typedef struct tc_dec_plan {
    uint32_t scaled, tw, th, climit, drop_alpha;
} tc_dec_plan;
/* a frame's plan from its header: TC_OK or the frame's status */
typedef int32_t (*tc_plan_fn)(const void* ctx, const tc_hdr* h, tc_dec_plan* plan);
void tc_plan_full(tc_dec_plan* p);
void tc_apply_plan_info(const tc_dec_plan* plan, const tc_hdr* h, topos_frame_output* o);
/* The batch decode of tc_frame_decode_batch with a plan per frame (fn NULL =
 * full size): a packet failing its structural parse fails the call; a plan
 * that cannot be resolved fails the call in query mode (planes_out NULL) and
 * only its frame otherwise; returns the first nonzero frame status. */
int32_t tc_decode_batch_mode(const topos_batch_packet* packets, uint32_t count, uint16_t* const* planes_out,
                             const size_t* strides, topos_frame_output* infos, tc_plan_fn fn, const void* ctx);

/* encode job of one frame (validation as tc_frame_encode), its stats and the
 * public status of a per-frame result (tc_api.c) */
struct tcg_enc_frame;
struct tcg_enc_result;
int32_t tc_prepare_encode(const topos_frame_config* cfg, const topos_frame_input* in, struct tcg_enc_frame* jf,
                          uint32_t* slice_count, uint8_t* qp_base);
void tc_fill_enc_stats(topos_frame_stats* st, const struct tcg_enc_result* r, uint32_t slices, uint8_t qp);
int32_t tc_enc_result_status(int32_t rc, size_t need, size_t cap);
/* public status (and statistics on success) of one encoded frame, V7-R2 or V8 */
int32_t tc_finish_encode(const struct tcg_enc_frame* jf, struct tcg_enc_result* r, topos_frame_stats* stats,
                         uint32_t slices, uint8_t qp, size_t out_cap);
/* a V8 frame with a segment no tile owns (the reference's self-check rejects it) */
int tc_v8_orphans(const struct tcg_enc_frame* jf);

#endif /* TC_INTERNAL_H */
