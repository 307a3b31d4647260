/* tc_decode_req.c - decode delivery modes (scaled, reduced, requests) and
 * persistent decoder contexts, over the plan-aware batch decode of tc_api.c.
 *
 * Reference: native/src/codec/codec.c:9100-9170 (tc_frame_decode_scaled),
 * :9172-9206 (scale dimensions, coefficient limits), :9208-9364 (request
 * validation and resolution), :9378-9545 (tc_frame_decode_request),
 * :9547-9636 (tc_frame_decode_reduced), :9639-9810 (batch forms);
 * native/src/codec/decoder_ctx.c (contexts). The GPU decode has no host
 * worker pool or per-context scratch, so a context is a validated handle and
 * its calls are the stateless ones with the same checks and statuses.
 */
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/topos_codec.h"
#include "tc_internal.h"

/* reference: codec.c:9172-9194 */
TC_EXPORT int32_t tc_decode_scale_dimensions(uint32_t source_width, uint32_t source_height, tc_decode_scale scale,
                                             uint32_t* target_width, uint32_t* target_height)
{
    if (target_width == NULL || target_height == NULL || source_width == 0u || source_height == 0u ||
        (int32_t)scale < (int32_t)TC_DECODE_SCALE_FULL || scale > TC_DECODE_SCALE_EIGHTH) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "invalid decode scale dimensions");
    }
    static const uint32_t div[5] = {1u, 2u, 3u, 4u, 8u};
    const uint32_t d = div[scale];
    *target_width = (source_width + d - 1u) / d;
    *target_height = (source_height + d - 1u) / d;
    return TC_OK;
}

/* reference: codec.c:9196-9206: zigzag positions a fixed ratio keeps */
static uint32_t scale_coefficient_limit(uint32_t scale)
{
    static const uint32_t lim[5] = {63u, 24u, 16u, 10u, 4u};
    return scale <= 4u ? lim[scale] : 0u;
}

/* reference: codec.c:9208-9270 */
static int32_t request_validate(const topos_decode_request* r)
{
    if (r == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode request == NULL"); }
    if (r->struct_size != (uint32_t)sizeof(topos_decode_request) || r->abi_version != TOPOS_CODEC_ABI_VERSION) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode request struct_size/abi_version");
    }
    if (r->mode > TC_DECODE_MODE_AUTO_2K || r->quality > TC_DECODE_QUALITY_HIGH ||
        (r->memory_type != TC_DECODE_MEMORY_CPU && r->memory_type != TC_DECODE_MEMORY_HOST_VISIBLE_GPU) ||
        (r->flags & ~TC_DECODE_FLAG_DROP_ALPHA) != 0u) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode request enum/flags invalid");
    }
    for (uint32_t i = 0; i < 4u; ++i) {
        if (r->reserved[i] != 0u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode request reserved nonzero"); }
    }
    if ((r->target_width == 0u) != (r->target_height == 0u)) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode request target width/height must be paired");
    }
    switch (r->mode) {
    case TC_DECODE_MODE_FULL:
        if (r->scale != TC_DECODE_SCALE_FULL || r->target_width != 0u || r->target_height != 0u) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "full decode request has target/scale");
        }
        break;
    case TC_DECODE_MODE_SCALED:
        if (r->scale != TC_DECODE_SCALE_FULL || r->target_width == 0u) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "scaled decode request requires target");
        }
        break;
    case TC_DECODE_MODE_REDUCED:
        if (r->scale > TC_DECODE_SCALE_EIGHTH) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "reduced decode request scale invalid");
        }
        if (r->target_width != 0u || r->target_height != 0u) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "reduced decode request does not accept target");
        }
        break;
    default: /* AUTO_2K */
        if (r->scale != TC_DECODE_SCALE_FULL) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "auto2k decode request scale invalid");
        }
        break;
    }
    return TC_OK;
}

/* reference: codec.c:9272-9364: the delivered grid of one frame */
static int32_t request_resolve(const void* ctx, const tc_hdr* h, tc_dec_plan* plan)
{
    const topos_decode_request* r = (const topos_decode_request*)ctx;
    int32_t rc = request_validate(r);
    if (rc != TC_OK) { return rc; }
    tc_plan_full(plan);
    plan->drop_alpha = (r->flags & TC_DECODE_FLAG_DROP_ALPHA) != 0u && h->amode != 0u;
    const uint32_t sw = h->vw, sh = h->vh;
    plan->tw = sw;
    plan->th = sh;
    switch (r->mode) {
    case TC_DECODE_MODE_FULL:
        return TC_OK;
    case TC_DECODE_MODE_SCALED:
        plan->tw = r->target_width;
        plan->th = r->target_height;
        plan->scaled = 1u;
        break;
    case TC_DECODE_MODE_REDUCED:
        rc = tc_decode_scale_dimensions(sw, sh, (tc_decode_scale)r->scale, &plan->tw, &plan->th);
        if (rc != TC_OK) { return rc; }
        plan->scaled = r->scale != TC_DECODE_SCALE_FULL;
        plan->climit = scale_coefficient_limit(r->scale);
        break;
    default: /* AUTO_2K */
        if (r->target_width != 0u) {
            plan->tw = r->target_width;
            plan->th = r->target_height;
            plan->scaled = plan->tw != sw || plan->th != sh;
            break;
        }
        if (sw <= 2048u && sh <= 2048u) { return TC_OK; }
        for (uint32_t s = TC_DECODE_SCALE_HALF; s <= TC_DECODE_SCALE_EIGHTH; ++s) {
            uint32_t tw = 0, th = 0;
            rc = tc_decode_scale_dimensions(sw, sh, (tc_decode_scale)s, &tw, &th);
            if (rc != TC_OK) { return rc; }
            if (tw <= 2048u && th <= 2048u) {
                plan->tw = tw;
                plan->th = th;
                plan->scaled = 1u;
                plan->climit = scale_coefficient_limit(s);
                break;
            }
        }
        break;
    }
    if (plan->tw == 0u || plan->th == 0u || plan->tw > sw || plan->th > sh || plan->tw > 65535u || plan->th > 65535u) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode target %ux%u exceeds source %ux%u", plan->tw, plan->th, sw, sh);
    }
    return TC_OK;
}

typedef struct fixed_plan {
    uint32_t scaled, tw, th, climit, scale;
} fixed_plan;

/* target size given by the caller (tc_frame_decode_scaled), all coefficients */
static int32_t scaled_resolve(const void* ctx, const tc_hdr* h, tc_dec_plan* plan)
{
    const fixed_plan* f = (const fixed_plan*)ctx;
    tc_plan_full(plan);
    if (f->tw > h->vw || f->th > h->vh || f->tw > 65535u || f->th > 65535u) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "scaled target %ux%u exceeds source %ux%u", f->tw, f->th, h->vw, h->vh);
    }
    plan->scaled = 1u;
    plan->tw = f->tw;
    plan->th = f->th;
    return TC_OK;
}

/* a context batch without a request: full size, reported as a resolved plan
 * (reference decoder_ctx.c:160-167 and 704-728) */
static int32_t full_resolve(const void* ctx, const tc_hdr* h, tc_dec_plan* plan)
{
    (void)ctx;
    tc_plan_full(plan);
    plan->tw = h->vw;
    plan->th = h->vh;
    return TC_OK;
}

/* fixed ratio of the source (tc_frame_decode_reduced and its batch form) */
static int32_t reduced_resolve(const void* ctx, const tc_hdr* h, tc_dec_plan* plan)
{
    const fixed_plan* f = (const fixed_plan*)ctx;
    tc_plan_full(plan);
    if (f->scale == TC_DECODE_SCALE_FULL) { return TC_OK; }
    const int32_t rc = tc_decode_scale_dimensions(h->vw, h->vh, (tc_decode_scale)f->scale, &plan->tw, &plan->th);
    if (rc != TC_OK) { return rc; }
    plan->scaled = 1u;
    plan->climit = scale_coefficient_limit(f->scale);
    return TC_OK;
}

static int32_t decode_one(const uint8_t* data, size_t size, uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                          const size_t strides[TC_FRAME_MAX_PLANES], topos_frame_output* o, tc_plan_fn fn,
                          const void* ctx)
{
    const topos_batch_packet one = {data, size};
    uint16_t* planes[TC_FRAME_MAX_PLANES] = {NULL, NULL, NULL, NULL};
    size_t st[TC_FRAME_MAX_PLANES] = {0u, 0u, 0u, 0u};
    for (uint32_t p = 0; p < TC_FRAME_MAX_PLANES && planes_out != NULL; ++p) {
        planes[p] = planes_out[p];
        st[p] = strides != NULL ? strides[p] : 0u;
    }
    return tc_decode_batch_mode(&one, 1u, planes_out != NULL ? planes : NULL, st, o, fn, ctx);
}

static int32_t info_reset(topos_frame_output* o)
{
    if (o == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "out_info == NULL"); }
    memset(o, 0, sizeof(*o));
    o->struct_size = (uint32_t)sizeof(topos_frame_output);
    o->abi_version = TOPOS_CODEC_ABI_VERSION;
    return TC_OK;
}

/* reference: codec.c:9378-9545 */
TC_EXPORT int32_t tc_frame_decode_request(const uint8_t* data, size_t size, const topos_decode_request* request,
                                          uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                                          const size_t strides[TC_FRAME_MAX_PLANES], topos_frame_output* out_info)
{
    int32_t rc = info_reset(out_info);
    if (rc != TC_OK) { return rc; }
    if (data == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "data == NULL"); }
    rc = request_validate(request);
    if (rc != TC_OK) { return rc; }
    if (tc_packet_major(data, size) == 8) {
        /* V8 (codec.c:9469-9482): the query and FULL decode; no scaled path */
        if (planes_out != NULL && request->mode != TC_DECODE_MODE_FULL) {
            rc = tc_v8_frame_decode(data, size, NULL, NULL, out_info);
            return rc != TC_OK ? rc : tc_fail(TC_ERR_NOT_IMPLEMENTED, "v8 reduced/auto2k path not defined");
        }
        return tc_v8_frame_decode(data, size, planes_out, strides, out_info);
    }
    return decode_one(data, size, planes_out, strides, out_info, request_resolve, request);
}

/* reference: codec.c:9100-9170 */
TC_EXPORT int32_t tc_frame_decode_scaled(const uint8_t* data, size_t size, uint32_t target_width,
                                         uint32_t target_height, uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                                         const size_t strides[TC_FRAME_MAX_PLANES], topos_frame_output* out_info)
{
    int32_t rc = info_reset(out_info);
    if (rc != TC_OK) { return rc; }
    if (data == NULL || target_width == 0u || target_height == 0u) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "scaled decode invalid arguments");
    }
    if (tc_packet_major(data, size) == 8) {
        /* V8 (codec.c:9123-9130): structure and information, no scaled path */
        rc = tc_v8_frame_decode(data, size, NULL, NULL, out_info);
        return rc != TC_OK ? rc : tc_fail(TC_ERR_NOT_IMPLEMENTED, "v8 scaled decode lands in format-plan batch 3");
    }
    const fixed_plan f = {1u, target_width, target_height, 63u, 0u};
    return decode_one(data, size, planes_out, strides, out_info, scaled_resolve, &f);
}

/* reference: codec.c:9547-9636 */
TC_EXPORT int32_t tc_frame_decode_reduced(const uint8_t* data, size_t size, tc_decode_scale scale,
                                          uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                                          const size_t strides[TC_FRAME_MAX_PLANES], topos_frame_output* out_info)
{
    if (out_info == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "out_info == NULL"); }
    if (scale == TC_DECODE_SCALE_FULL) { return tc_frame_decode(data, size, planes_out, strides, out_info); }
    if (data == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "data == NULL"); }
    if ((int32_t)scale < 0 || scale > TC_DECODE_SCALE_EIGHTH) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "invalid decode scale dimensions");
    }
    /* out_info is written only once the packet's structure parses
     * (codec.c:9602-9612); a V8 packet fails that parse */
    const fixed_plan f = {1u, 0u, 0u, 63u, (uint32_t)scale};
    return decode_one(data, size, planes_out, strides, out_info, reduced_resolve, &f);
}

/* reference: codec.c:9639-9665, 9807-9815 */
TC_EXPORT int32_t tc_frame_decode_batch_reduced(const topos_batch_packet* packets, uint32_t count,
                                                tc_decode_scale scale, uint16_t* const* planes_out,
                                                const size_t* strides, topos_frame_output* infos)
{
    if (count == 0u) { return TC_OK; }
    if (count > TC_BATCH_MAX_FRAMES) { return tc_fail(TC_ERR_LIMIT_EXCEEDED, "batch count %u > %u", count, TC_BATCH_MAX_FRAMES); }
    if (infos == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "infos == NULL"); }
    if (packets == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "batch packets == NULL"); }
    if ((int32_t)scale < 0 || scale > TC_DECODE_SCALE_EIGHTH) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "invalid decode scale %u", (unsigned)scale);
    }
    const fixed_plan f = {1u, 0u, 0u, 63u, (uint32_t)scale};
    return tc_decode_batch_mode(packets, count, planes_out, strides, infos, reduced_resolve, &f);
}

/* ------------------------------------------------------------ decoder contexts */

struct tc_decoder {
    uint32_t magic;
    _Atomic uint32_t max_slice_workers; /* kept for the reference's contract */
};

#define TC_DECODER_MAGIC 0x54444543u

static int decoder_valid(const tc_decoder* d) { return d != NULL && d->magic == TC_DECODER_MAGIC; }

/* reference: decoder_ctx.c:38-66 */
TC_EXPORT int32_t tc_decoder_create(const topos_decoder_config* cfg, tc_decoder** out)
{
    if (out == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "out == NULL"); }
    *out = NULL;
    if (cfg != NULL && (cfg->struct_size != (uint32_t)sizeof(topos_decoder_config) ||
                        cfg->abi_version != TOPOS_CODEC_ABI_VERSION)) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decoder config struct_size/abi_version");
    }
    tc_decoder* d = (tc_decoder*)calloc(1, sizeof(tc_decoder));
    if (d == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "decoder context"); }
    atomic_init(&d->max_slice_workers, cfg != NULL ? cfg->max_slice_workers : 0u);
    d->magic = TC_DECODER_MAGIC;
    *out = d;
    return TC_OK;
}

/* reference: decoder_ctx.c:68-78 */
TC_EXPORT int32_t tc_decoder_set_max_slice_workers(tc_decoder* dec, uint32_t workers)
{
    if (!decoder_valid(dec)) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "decoder handle invalid"); }
    atomic_store(&dec->max_slice_workers, workers);
    return TC_OK;
}

/* reference: decoder_ctx.c:80-89 */
TC_EXPORT void tc_decoder_destroy(tc_decoder* dec)
{
    if (!decoder_valid(dec)) { return; }
    dec->magic = 0u;
    free(dec);
}

/* reference: decoder_ctx.c:169-195 */
TC_EXPORT int32_t tc_decoder_prepare(tc_decoder* dec, const uint8_t* packet, size_t size, topos_frame_output* info)
{
    if (!decoder_valid(dec)) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "decoder handle invalid"); }
    if (info == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "info == NULL"); }
    if (packet == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "packet == NULL"); }
    return tc_frame_decode(packet, size, NULL, NULL, info);
}

/* reference: decoder_ctx.c:197-233 */
TC_EXPORT int32_t tc_decoder_prepare_request(tc_decoder* dec, const uint8_t* packet, size_t size,
                                             const topos_decode_request* request, topos_frame_output* info)
{
    if (!decoder_valid(dec)) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "decoder handle invalid"); }
    if (info == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "info == NULL"); }
    (void)info_reset(info);
    if (packet == NULL || request == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode request arguments invalid"); }
    return decode_one(packet, size, NULL, NULL, info, request_resolve, request);
}

/* plane views of a frame as pointers; an invalid view leaves its plane NULL,
 * which fails the frame as an invalid argument */
static void views_to_planes(const topos_plane_view* out, uint16_t** planes, size_t* strides)
{
    for (uint32_t p = 0; p < TC_FRAME_MAX_PLANES; ++p) {
        const topos_plane_view* v = &out[p];
        const int ok = v->struct_size == (uint32_t)sizeof(topos_plane_view) && v->abi_version == TOPOS_CODEC_ABI_VERSION;
        planes[p] = ok ? v->pixels : NULL;
        strides[p] = ok ? v->stride : 0u;
    }
}

static int32_t decoder_decode_one(tc_decoder* dec, const uint8_t* packet, size_t size,
                                  const topos_decode_request* request, const topos_plane_view* out,
                                  topos_frame_output* info)
{
    if (!decoder_valid(dec)) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "decoder handle invalid"); }
    if (info == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "info == NULL"); }
    if (packet == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "packet == NULL"); }
    if (out == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "out == NULL"); }
    (void)info_reset(info);
    if (request != NULL) {
        const int32_t rc = request_validate(request);
        if (rc != TC_OK) { return rc; }
    }
    uint16_t* planes[TC_FRAME_MAX_PLANES];
    size_t strides[TC_FRAME_MAX_PLANES];
    views_to_planes(out, planes, strides);
    return decode_one(packet, size, planes, strides, info, request != NULL ? request_resolve : NULL, request);
}

/* reference: decoder_ctx.c:235-334 */
TC_EXPORT int32_t tc_decoder_decode(tc_decoder* dec, const uint8_t* packet, size_t size,
                                    const topos_plane_view out[TC_FRAME_MAX_PLANES], topos_frame_output* info)
{
    return decoder_decode_one(dec, packet, size, NULL, out, info);
}

/* reference: decoder_ctx.c:336-466 */
TC_EXPORT int32_t tc_decoder_decode_request(tc_decoder* dec, const uint8_t* packet, size_t size,
                                            const topos_decode_request* request,
                                            const topos_plane_view out[TC_FRAME_MAX_PLANES], topos_frame_output* info)
{
    if (decoder_valid(dec) && request == NULL) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "request decode arguments invalid");
    }
    return decoder_decode_one(dec, packet, size, request, out, info);
}

static int32_t decoder_batch(tc_decoder* dec, const topos_batch_packet* packets, uint32_t count,
                             const topos_decode_request* request, const topos_plane_view* out,
                             topos_frame_output* infos)
{
    if (!decoder_valid(dec)) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "decoder handle invalid"); }
    if (count == 0u) { return TC_OK; }
    if (request != NULL) {
        const int32_t rc = request_validate(request);
        if (rc != TC_OK) { return rc; }
    }
    if (count > TC_BATCH_MAX_FRAMES) { return tc_fail(TC_ERR_LIMIT_EXCEEDED, "batch count %u > %u", count, TC_BATCH_MAX_FRAMES); }
    tc_plan_fn fn = request != NULL ? request_resolve : full_resolve;
    if (out == NULL) { return tc_decode_batch_mode(packets, count, NULL, NULL, infos, fn, request); }
    uint16_t** planes = (uint16_t**)malloc(sizeof(uint16_t*) * (size_t)count * TC_FRAME_MAX_PLANES);
    size_t* strides = (size_t*)malloc(sizeof(size_t) * (size_t)count * TC_FRAME_MAX_PLANES);
    if (planes == NULL || strides == NULL) {
        free(planes);
        free(strides);
        return tc_fail(TC_ERR_OUT_OF_MEMORY, "decoder batch views");
    }
    for (uint32_t i = 0; i < count; ++i) {
        views_to_planes(out + (size_t)i * TC_FRAME_MAX_PLANES, planes + (size_t)i * TC_FRAME_MAX_PLANES,
                        strides + (size_t)i * TC_FRAME_MAX_PLANES);
    }
    const int32_t rc = tc_decode_batch_mode(packets, count, planes, strides, infos, fn, request);
    free(planes);
    free(strides);
    return rc;
}

/* reference: decoder_ctx.c:736-753 */
TC_EXPORT int32_t tc_decoder_decode_batch(tc_decoder* dec, const topos_batch_packet* packets, uint32_t count,
                                          const topos_plane_view* out, topos_frame_output* infos)
{
    return decoder_batch(dec, packets, count, NULL, out, infos);
}

TC_EXPORT int32_t tc_decoder_decode_batch_request(tc_decoder* dec, const topos_batch_packet* packets, uint32_t count,
                                                  const topos_decode_request* request, const topos_plane_view* out,
                                                  topos_frame_output* infos)
{
    return decoder_batch(dec, packets, count, request, out, infos);
}

/* reference: decoder_ctx.c:468-506 */
TC_EXPORT int32_t tc_decoder_decode_surface(tc_decoder* dec, const uint8_t* packet, size_t size,
                                            const topos_decode_surface* surface, topos_frame_output* info)
{
    if (surface == NULL ||
        (surface->memory_type != TC_DECODE_MEMORY_CPU && surface->memory_type != TC_DECODE_MEMORY_HOST_VISIBLE_GPU)) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode surface invalid");
    }
    if (surface->struct_size != (uint32_t)sizeof(topos_decode_surface) || surface->abi_version != TOPOS_CODEC_ABI_VERSION) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode surface struct_size/abi_version");
    }
    return tc_decoder_decode(dec, packet, size, surface->planes, info);
}

TC_EXPORT int32_t tc_decoder_decode_surface_request(tc_decoder* dec, const uint8_t* packet, size_t size,
                                                    const topos_decode_request* request,
                                                    const topos_decode_surface* surface, topos_frame_output* info)
{
    if (surface == NULL ||
        (surface->memory_type != TC_DECODE_MEMORY_CPU && surface->memory_type != TC_DECODE_MEMORY_HOST_VISIBLE_GPU)) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode surface invalid");
    }
    if (surface->struct_size != (uint32_t)sizeof(topos_decode_surface) || surface->abi_version != TOPOS_CODEC_ABI_VERSION ||
        request == NULL) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "decode surface request invalid");
    }
    if (request->memory_type != surface->memory_type) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "request/surface memory_type mismatch");
    }
    return tc_decoder_decode_request(dec, packet, size, request, surface->planes, info);
}
