/* topos_codec_compat.h - entry points of the reference ABI that lie outside the
 * GPU intra frame path. The reference's Python binding binds them when it
 * loads the library (reference: python/topos_codec/topos_binding.py,
 * ToposCodec._configure_signatures), so this library exports them with the
 * reference's parameter lists. Each returns TC_ERR_NOT_IMPLEMENTED (void ones
 * do nothing), except where the comment says otherwise. Handle and record
 * types the path does not use are left incomplete here; enum parameters are
 * passed as int32_t, which is how the reference ABI passes them.
 */
#ifndef TOPOS_CODEC_COMPAT_H
#define TOPOS_CODEC_COMPAT_H

#include "topos_codec.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct topos_gop_context topos_gop_context;
typedef struct topos_mux topos_mux;
typedef struct topos_gop_frame_info topos_gop_frame_info;
typedef struct topos_movie_config topos_movie_config;
typedef struct topos_timecode_info topos_timecode_info;
typedef struct topos_audio_track_config topos_audio_track_config;
typedef struct topos_audio_track_info topos_audio_track_info;

/* reference: native/include/topos_codec.h:122. Implemented: "experimental",
 * "reference", "eligible", "default" for 0..3, "unknown" otherwise. */
const char* tc_scalable_status_name(int32_t status);

/* reference: native/src/common/tpool.h:44-45. The GPU path has no host thread
 * pool: the setter is ignored and the count reads 1. */
void tc_dev_set_thread_count(int32_t n);
int32_t tc_dev_thread_count(void);

/* reference: native/src/codec/codec.h:213, 246, 487-494 (development
 * statistics). Resets do nothing; the histogram getters write zeros
 * (dc 29, run 64, lvl 28 counts; pair histogram 64 x 28). */
void tc_dev_decode_stats_reset(void);
void tc_dev_encode_stats_reset(void);
void tc_dev_symbol_hist_reset(void);
void tc_dev_symbol_hist_get(uint64_t* dc, uint64_t* run, uint64_t* lvl);
void tc_dev_symbol_pair_hist_get(uint32_t plane, uint64_t* pair_hist);

/* reference: native/include/topos_codec.h:316-328, native/src/codec/codec.c:7789
 * (size-targeted encode). Implemented: the reference's deterministic qp
 * searches (strict by default: the smallest qp in [qp_min, qp_max] whose
 * packet fits target_bytes; the legacy linear and "r6" searches by
 * TOPOS_SIZED_SEARCH or tc_dev_set_sized_mode) over exact packet sizes that
 * the GPU encodes a window of qps at a time; the packet, stats, qp_used and
 * every status equal the reference's for the same call sequence. qp_min >
 * qp_max or either above 95 is TC_ERR_INVALID_ARGUMENT; a target no qp meets
 * returns the qp_max packet (best effort); out is written only on TC_OK and
 * a final packet larger than out_cap is TC_ERR_BUFFER_TOO_SMALL with its size
 * in stats. */
int32_t tc_frame_encode_sized(const topos_frame_config* cfg, const topos_frame_input* input, uint32_t target_bytes,
                              uint8_t qp_min, uint8_t qp_max, uint8_t* qp_used, uint8_t* out, size_t out_cap,
                              topos_frame_stats* stats);

/* reference: native/src/codec/codec.c:7110-7178 (developer switches of the
 * size-targeted encode). Implemented: the search mode (0 strict, 1 linear,
 * 2 r6; other values select strict; overrides TOPOS_SIZED_SEARCH), the legacy
 * two-valued form, turning off the cross-call qp hint or its two-point model,
 * turning off the exact-count probe (the strict search then falls back to the
 * linear one), and the counters of calls and probe encodes. */
void tc_dev_set_sized_mode(int32_t mode);
void tc_dev_set_sized_search(int legacy);
void tc_dev_set_qp_hint(int disable);
void tc_dev_set_qp_hint_model(int disable);
void tc_dev_set_sized_m7(int disable);
void tc_dev_sized_reset(void);
uint64_t tc_dev_sized_iters(void);
uint64_t tc_dev_sized_calls(void);
/* reference: native/include/topos_codec.h:613-646 (GOP / P-frame context) */
void tc_gop_context_close(topos_gop_context* ctx);
int32_t tc_gop_context_observe(topos_gop_context* ctx, const uint8_t* data, size_t size, topos_gop_frame_info* info);
int32_t tc_gop_context_feed(topos_gop_context* ctx, const uint8_t* data, size_t size, const topos_plane_view* out,
                            topos_gop_frame_info* info);
int32_t tc_gop_context_encode_frame(topos_gop_context* ctx, const topos_frame_input* input, uint8_t* out,
                                    size_t out_cap, size_t* need_size, int force_intra, topos_frame_stats* stats);
void tc_gop_context_abort(topos_gop_context* ctx, int reset_to_i);
int32_t tc_gop_context_state(topos_gop_context* ctx, uint32_t* out_state, uint16_t* out_gop_id);

/* reference: native/include/topos_codec.h:833-943 (MOV writer) */
int32_t tc_mux_create(const topos_movie_config* cfg, const topos_io* sink, topos_mux** out);
int32_t tc_mux_add_packet(topos_mux* mux, const uint8_t* packet, size_t size, uint64_t pts_tick, uint32_t dur_tick);
int32_t tc_mux_set_alpha_budget(topos_mux* mux, const topos_alpha_budget_info* info);
int32_t tc_mux_add_audio(topos_mux* mux, const uint8_t* data, size_t size, uint32_t num_samples);
int32_t tc_mux_set_audio_asc(topos_mux* mux, const uint8_t* asc, size_t size);
int32_t tc_mux_set_timecode(topos_mux* mux, uint32_t hh, uint32_t mm, uint32_t ss, uint32_t ff, uint32_t fps,
                            uint32_t drop_frame);
int32_t tc_mux_set_audio_priming(topos_mux* mux, uint32_t samples);
int32_t tc_mux_finish(topos_mux* mux);
void tc_mux_free(topos_mux* mux);
int32_t tc_mux_add_audio_track(topos_mux* mux, const topos_audio_track_config* cfg);
int32_t tc_mux_set_audio_track_asc(topos_mux* mux, uint32_t track, const uint8_t* asc, size_t size);
int32_t tc_mux_set_audio_track_priming(topos_mux* mux, uint32_t track, uint32_t samples);
int32_t tc_mux_add_audio_to(topos_mux* mux, uint32_t track, const uint8_t* data, size_t size, uint32_t num_samples);

/* reference: native/include/topos_codec.h:880-1014 (MOV reader) */
int32_t tc_movie_faststart(const topos_io* src, const topos_io* dst);
int32_t tc_movie_audio_info(const topos_movie* movie, topos_audio_track_info* info);
int32_t tc_movie_audio_track_count(const topos_movie* movie, uint32_t* out_count);
int32_t tc_movie_audio_info_at(const topos_movie* movie, uint32_t track, topos_audio_track_info* info);
int32_t tc_movie_read_audio_at(const topos_movie* movie, uint32_t track, uint64_t start_chunk, uint32_t chunk_count,
                               uint8_t* buf, size_t cap, size_t* need_size);
int32_t tc_movie_timecode(const topos_movie* movie, topos_timecode_info* out);
int32_t tc_movie_read_audio(const topos_movie* movie, uint64_t start_chunk, uint32_t chunk_count, uint8_t* buf,
                            size_t cap, size_t* need_size);

#ifdef __cplusplus
}
#endif

#endif /* TOPOS_CODEC_COMPAT_H */
