/* tc_stubs.c - exports of the reference ABI outside the GPU intra path
 * (declarations and reference citations in include/topos_codec_compat.h).
 * They exist so that the reference's Python binding, which binds every one of
 * them when it loads a library, can load this one and run the frame path. */
#include <string.h>

#include "../../../include/topos_codec_compat.h"
#include "tc_internal.h"

#define NOT_PATH(name) tc_fail(TC_ERR_NOT_IMPLEMENTED, "%s is not part of the GPU intra frame path", name)

TC_EXPORT const char* tc_scalable_status_name(int32_t status)
{
    switch (status) {
    case 0: return "experimental";
    case 1: return "reference";
    case 2: return "eligible";
    case 3: return "default";
    default: return "unknown";
    }
}

TC_EXPORT void tc_dev_set_thread_count(int32_t n) { (void)n; }
TC_EXPORT int32_t tc_dev_thread_count(void) { return 1; }
TC_EXPORT void tc_dev_decode_stats_reset(void) {}
TC_EXPORT void tc_dev_encode_stats_reset(void) {}
TC_EXPORT void tc_dev_symbol_hist_reset(void) {}

TC_EXPORT void tc_dev_symbol_hist_get(uint64_t* dc, uint64_t* run, uint64_t* lvl)
{
    if (dc != NULL) { memset(dc, 0, 29u * sizeof(uint64_t)); }
    if (run != NULL) { memset(run, 0, 64u * sizeof(uint64_t)); }
    if (lvl != NULL) { memset(lvl, 0, 28u * sizeof(uint64_t)); }
}

TC_EXPORT void tc_dev_symbol_pair_hist_get(uint32_t plane, uint64_t* pair_hist)
{
    (void)plane;
    if (pair_hist != NULL) { memset(pair_hist, 0, 64u * 28u * sizeof(uint64_t)); }
}

TC_EXPORT void tc_gop_context_close(topos_gop_context* ctx) { (void)ctx; }

TC_EXPORT int32_t tc_gop_context_observe(topos_gop_context* ctx, const uint8_t* data, size_t size,
                                         topos_gop_frame_info* info)
{
    (void)ctx; (void)data; (void)size; (void)info;
    return NOT_PATH("tc_gop_context_observe");
}

TC_EXPORT int32_t tc_gop_context_feed(topos_gop_context* ctx, const uint8_t* data, size_t size,
                                      const topos_plane_view* out, topos_gop_frame_info* info)
{
    (void)ctx; (void)data; (void)size; (void)out; (void)info;
    return NOT_PATH("tc_gop_context_feed");
}

TC_EXPORT int32_t tc_gop_context_encode_frame(topos_gop_context* ctx, const topos_frame_input* input, uint8_t* out,
                                              size_t out_cap, size_t* need_size, int force_intra,
                                              topos_frame_stats* stats)
{
    (void)ctx; (void)input; (void)out; (void)out_cap; (void)need_size; (void)force_intra; (void)stats;
    return NOT_PATH("tc_gop_context_encode_frame");
}

TC_EXPORT void tc_gop_context_abort(topos_gop_context* ctx, int reset_to_i) { (void)ctx; (void)reset_to_i; }

TC_EXPORT int32_t tc_gop_context_state(topos_gop_context* ctx, uint32_t* out_state, uint16_t* out_gop_id)
{
    (void)ctx; (void)out_state; (void)out_gop_id;
    return NOT_PATH("tc_gop_context_state");
}

/* ---- MOV writer / reader ---- */

TC_EXPORT int32_t tc_mux_create(const topos_movie_config* cfg, const topos_io* sink, topos_mux** out)
{
    (void)cfg; (void)sink;
    if (out != NULL) { *out = NULL; }
    return NOT_PATH("tc_mux_create");
}

TC_EXPORT int32_t tc_mux_add_packet(topos_mux* mux, const uint8_t* packet, size_t size, uint64_t pts_tick,
                                    uint32_t dur_tick)
{
    (void)mux; (void)packet; (void)size; (void)pts_tick; (void)dur_tick;
    return NOT_PATH("tc_mux_add_packet");
}

TC_EXPORT int32_t tc_mux_set_alpha_budget(topos_mux* mux, const topos_alpha_budget_info* info)
{
    (void)mux; (void)info;
    return NOT_PATH("tc_mux_set_alpha_budget");
}

TC_EXPORT int32_t tc_mux_add_audio(topos_mux* mux, const uint8_t* data, size_t size, uint32_t num_samples)
{
    (void)mux; (void)data; (void)size; (void)num_samples;
    return NOT_PATH("tc_mux_add_audio");
}

TC_EXPORT int32_t tc_mux_set_audio_asc(topos_mux* mux, const uint8_t* asc, size_t size)
{
    (void)mux; (void)asc; (void)size;
    return NOT_PATH("tc_mux_set_audio_asc");
}

TC_EXPORT int32_t tc_mux_set_timecode(topos_mux* mux, uint32_t hh, uint32_t mm, uint32_t ss, uint32_t ff,
                                      uint32_t fps, uint32_t drop_frame)
{
    (void)mux; (void)hh; (void)mm; (void)ss; (void)ff; (void)fps; (void)drop_frame;
    return NOT_PATH("tc_mux_set_timecode");
}

TC_EXPORT int32_t tc_mux_set_audio_priming(topos_mux* mux, uint32_t samples)
{
    (void)mux; (void)samples;
    return NOT_PATH("tc_mux_set_audio_priming");
}

TC_EXPORT int32_t tc_mux_finish(topos_mux* mux)
{
    (void)mux;
    return NOT_PATH("tc_mux_finish");
}

TC_EXPORT void tc_mux_free(topos_mux* mux) { (void)mux; }

TC_EXPORT int32_t tc_mux_add_audio_track(topos_mux* mux, const topos_audio_track_config* cfg)
{
    (void)mux; (void)cfg;
    return NOT_PATH("tc_mux_add_audio_track");
}

TC_EXPORT int32_t tc_mux_set_audio_track_asc(topos_mux* mux, uint32_t track, const uint8_t* asc, size_t size)
{
    (void)mux; (void)track; (void)asc; (void)size;
    return NOT_PATH("tc_mux_set_audio_track_asc");
}

TC_EXPORT int32_t tc_mux_set_audio_track_priming(topos_mux* mux, uint32_t track, uint32_t samples)
{
    (void)mux; (void)track; (void)samples;
    return NOT_PATH("tc_mux_set_audio_track_priming");
}

TC_EXPORT int32_t tc_mux_add_audio_to(topos_mux* mux, uint32_t track, const uint8_t* data, size_t size,
                                      uint32_t num_samples)
{
    (void)mux; (void)track; (void)data; (void)size; (void)num_samples;
    return NOT_PATH("tc_mux_add_audio_to");
}

TC_EXPORT int32_t tc_movie_faststart(const topos_io* src, const topos_io* dst)
{
    (void)src; (void)dst;
    return NOT_PATH("tc_movie_faststart");
}




TC_EXPORT int32_t tc_movie_audio_info(const topos_movie* movie, topos_audio_track_info* info)
{
    (void)movie; (void)info;
    return NOT_PATH("tc_movie_audio_info");
}

TC_EXPORT int32_t tc_movie_audio_track_count(const topos_movie* movie, uint32_t* out_count)
{
    (void)movie; (void)out_count;
    return NOT_PATH("tc_movie_audio_track_count");
}

TC_EXPORT int32_t tc_movie_audio_info_at(const topos_movie* movie, uint32_t track, topos_audio_track_info* info)
{
    (void)movie; (void)track; (void)info;
    return NOT_PATH("tc_movie_audio_info_at");
}

TC_EXPORT int32_t tc_movie_read_audio_at(const topos_movie* movie, uint32_t track, uint64_t start_chunk,
                                         uint32_t chunk_count, uint8_t* buf, size_t cap, size_t* need_size)
{
    (void)movie; (void)track; (void)start_chunk; (void)chunk_count; (void)buf; (void)cap; (void)need_size;
    return NOT_PATH("tc_movie_read_audio_at");
}

TC_EXPORT int32_t tc_movie_timecode(const topos_movie* movie, topos_timecode_info* out)
{
    (void)movie; (void)out;
    return NOT_PATH("tc_movie_timecode");
}

TC_EXPORT int32_t tc_movie_read_audio(const topos_movie* movie, uint64_t start_chunk, uint32_t chunk_count,
                                      uint8_t* buf, size_t cap, size_t* need_size)
{
    (void)movie; (void)start_chunk; (void)chunk_count; (void)buf; (void)cap; (void)need_size;
    return NOT_PATH("tc_movie_read_audio");
}





