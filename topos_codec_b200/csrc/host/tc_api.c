/* tc_api.c - public entry points of the B200 Topos Codec library (C11).
 *
 * Semantics follow the reference entry points they replace (cited per
 * function); all per-pixel and per-symbol work runs on the GPU through
 * tcg_device.h. There is no CPU coding path: without a CUDA device the frame
 * functions fail with TC_ERR_NOT_IMPLEMENTED and a detail message.
 */
#include <stdlib.h>
#include <string.h>

#include "../tcg_device.h"
#include "tc_internal.h"

#define TC_VERSION_MAJOR 0
#define TC_VERSION_MINOR 1
#define TC_VERSION_PATCH 0

/* reference: native/src/version.c:8-28 */
TC_EXPORT int32_t tc_abi_version(void) { return TOPOS_CODEC_ABI_VERSION; }

TC_EXPORT int32_t tc_version(topos_version_info* out)
{
    if (out == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "tc_version: out is NULL"); }
    out->struct_size = (uint32_t)sizeof(topos_version_info);
    out->abi_version = TOPOS_CODEC_ABI_VERSION;
    out->version_major = TC_VERSION_MAJOR;
    out->version_minor = TC_VERSION_MINOR;
    out->version_patch = TC_VERSION_PATCH;
    out->git_commit = "b200";
    out->build_target = "sm_100a-cuda";
    return TC_OK;
}

/* reference: native/src/version.c:30-40 */
TC_EXPORT int32_t tc_query_cpu_features(topos_cpu_features* out)
{
    if (out == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "tc_query_cpu_features: out is NULL"); }
    out->struct_size = (uint32_t)sizeof(topos_cpu_features);
    out->abi_version = TOPOS_CODEC_ABI_VERSION;
    uint32_t f = 0;
#if defined(__x86_64__)
    __builtin_cpu_init();
    if (__builtin_cpu_supports("avx2")) { f |= TOPOS_CPU_X86_AVX2; }
    if (__builtin_cpu_supports("avx512f")) { f |= TOPOS_CPU_X86_AVX512F; }
    if (__builtin_cpu_supports("fma")) { f |= TOPOS_CPU_X86_FMA; }
#elif defined(__aarch64__)
    f |= TOPOS_CPU_ARM_NEON;
#endif
    out->flags = f;
    return TC_OK;
}

/* reference: native/src/version.c:42-62; advertises the paths implemented here */
TC_EXPORT int32_t tc_query_capabilities(topos_codec_capabilities* out)
{
    if (out == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "tc_query_capabilities: out is NULL"); }
    out->struct_size = (uint32_t)sizeof(topos_codec_capabilities);
    out->abi_version = TOPOS_CODEC_ABI_VERSION;
    out->flags = TC_CODEC_CAP_FULL_DECODE | TC_CODEC_CAP_CPU_SURFACE_OUTPUT;
    out->max_width = TC_CODEC_MAX_DIM;
    out->max_height = TC_CODEC_MAX_DIM;
    out->auto2k_max_dim = TC_CODEC_AUTO_2K_MAX_DIM;
    return TC_OK;
}

/* reference: native/src/version.c:90-146 */
TC_EXPORT int32_t tc_query_support(uint32_t profile, uint32_t pf, uint32_t bd, uint32_t am)
{
    if (profile != 3u && profile != 5u && profile != 6u && profile != 7u) {
        return tc_fail(TC_ERR_UNSUPPORTED_PROFILE, "profile %u not in {3,5,6,7}", profile);
    }
    if (pf > 3u || (bd != 10u && bd != 12u && bd != 16u)) {
        return tc_fail(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "pixel_format %u / bit_depth %u unsupported", pf, bd);
    }
    if ((profile == 7u) != (pf == 3u)) {
        return tc_fail(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "profile 7 requires pixel_format 3 and vice versa");
    }
    if (profile == 7u && bd != 12u && bd != 16u) { return tc_fail(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "profile 7 requires 12/16-bit"); }
    if (profile == 7u && am != 0u) { return tc_fail(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "profile 7 requires no alpha"); }
    if ((profile == 5u || profile == 6u) && pf == 0u) {
        return tc_fail(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "profile %u requires 4:4:4", profile);
    }
    if (profile == 6u && bd != 12u) { return tc_fail(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "profile 6 requires 12-bit"); }
    if (am > 2u) { return tc_fail(TC_ERR_UNSUPPORTED_ALPHA_MODE, "alpha_mode %u > 2", am); }
    return TC_OK;
}

/* reference: native/src/codec/codec.c:426-605 */
TC_EXPORT int32_t tc_frame_config_validate(const topos_frame_config* c)
{
    if (c == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "cfg == NULL"); }
    if (c->struct_size != 0u && c->struct_size != (uint32_t)sizeof(topos_frame_config)) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "cfg struct_size %u != %u", c->struct_size, (unsigned)sizeof(topos_frame_config));
    }
    if (c->abi_version != 0u && c->abi_version != (uint32_t)TOPOS_CODEC_ABI_VERSION) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "cfg abi_version %u unsupported", c->abi_version);
    }
    if (c->visible_width == 0u || c->visible_height == 0u || c->visible_width > TC_MAX_DIM || c->visible_height > TC_MAX_DIM) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "visible %ux%u out of 1..16384", c->visible_width, c->visible_height);
    }
    if (c->qp_base > TC_QP_MAX) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "qp_base %u > 95", c->qp_base); }
    if (c->reserved[0] > 11u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "reserved[0] coding selection %u not in {0..11}", c->reserved[0]); }
    if (c->reserved[0] >= 2u && c->reserved[0] <= 7u) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "reserved[0] coding selection %u retired; write domain is {0,1,8,9,10}", c->reserved[0]);
    }
    if (c->reserved[1] > 1u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "reserved[1] AQ mode %u not in {0,1}", c->reserved[1]); }
    if (c->reserved[2] > 1u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "reserved[2] RDO mode %u not in {0,1}", c->reserved[2]); }
    {
        const uint8_t em = (uint8_t)(c->reserved[0] & 0xFFu);
        const int end = em >= 10u ? 6 : (em == 9u ? 5 : 3);
        for (int i = end; i < 8; ++i) {
            if (em == 8u && i == 5) { continue; }
            if (c->reserved[i] != 0u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "reserved[%d] must be 0 (got %u)", i, c->reserved[i]); }
        }
        if (em == 8u && c->reserved[5] != 0u) {
            if ((c->reserved[5] & ~3u) != 0u || c->profile != 3u || c->pixel_format != 0u || c->bit_depth != 10u) {
                return tc_fail(TC_ERR_INVALID_ARGUMENT, "reserved[5] output features %u require profile 3 / 4:2:2 / 10-bit", c->reserved[5]);
            }
        }
        if (em == 10u || em == 11u) {
            if (c->reserved[3] > 1u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "temporal frame_type %u not in {0,1}", c->reserved[3]); }
            if (c->reserved[5] != (c->reserved[3] == 0u ? 0u : 1u)) {
                return tc_fail(TC_ERR_INVALID_ARGUMENT, "temporal ref_distance %u for frame_type %u", c->reserved[5], c->reserved[3]);
            }
        }
    }
    if (c->alpha_mode > 2u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "alpha_mode %u > 2", c->alpha_mode); }
    if (c->alpha_mode == 1u && c->alpha_bit_depth != 16u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "lossless alpha requires bit_depth 16"); }
    if (c->alpha_mode == 2u && c->alpha_bit_depth != 8u && c->alpha_bit_depth != 10u && c->alpha_bit_depth != 12u) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "near-lossless alpha bit_depth %u not in {8,10,12}", c->alpha_bit_depth);
    }
    if (c->pixel_format == 3u) {
        if (c->alpha_mode != 0u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "TRAW (pixel_format=3) does not support alpha"); }
        if (c->qp_delta_chroma != 0) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "qp_delta_chroma must be 0 for TRAW"); }
    }
    tc_hdr h;
    tc_cfg_to_hdr(c, &h);
    int32_t rc = tc_hdr_geometry(&h);
    if (rc != TC_OK) { return rc; }
    rc = tc_band_plan(&h, tc_cfg_slice_rows(c), NULL);
    if (rc != TC_OK) { return rc; }
    h.slices = (uint16_t)(c->pixel_format == 3u ? 4u : 3u + (c->alpha_mode != 0u ? 1u : 0u));
    h.size = TC_HDR_SIZE;
    rc = tc_hdr_validate(&h);
    if (rc != TC_OK) { return rc; }
    if (c->bit_depth >= 13u && c->reserved[0] != 8u && c->reserved[0] != 9u) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "entropy mode %u is 12-bit frozen; bit_depth %u requires reserved[0] in {8,9}",
                       c->reserved[0], c->bit_depth);
    }
    return TC_OK;
}

/* reference: native/src/codec/codec.c:607-647 */
TC_EXPORT size_t tc_frame_packet_bound(const topos_frame_config* c)
{
    if (c == NULL || c->visible_width == 0u || c->visible_height == 0u || c->visible_width > TC_MAX_DIM ||
        c->visible_height > TC_MAX_DIM) {
        return 0u;
    }
    const uint64_t cw = (c->visible_width + 7u) / 8u * 8u, ch = (c->visible_height + 7u) / 8u * 8u;
    uint64_t ccw, cch;
    if (c->pixel_format == 0u) {
        ccw = (((uint64_t)c->visible_width + 1u) / 2u + 7u) / 8u * 8u; cch = ch;
    } else if (c->pixel_format == 3u) {
        ccw = (((uint64_t)c->visible_width + 1u) / 2u + 7u) / 8u * 8u;
        cch = (((uint64_t)c->visible_height + 1u) / 2u + 7u) / 8u * 8u;
    } else {
        ccw = cw; cch = ch;
    }
    const uint64_t blocks = c->pixel_format == 3u ? 4u * ((ccw * cch) / 64u) : (cw * ch) / 64u + 2u * ((ccw * cch) / 64u);
    const uint64_t planes = c->pixel_format == 3u ? 4u : 3u;
    uint64_t bound = 53u + planes * (17u + blocks * 1024u);
    if (c->alpha_mode != 0u) { bound += 17u + cw * ch * 16u; }
    return bound > TC_MAX_PACKET ? (size_t)TC_MAX_PACKET : (size_t)bound;
}

/* reference: native/src/codec/codec.c:9807-9831 */
TC_EXPORT int32_t tc_frame_plane_geometry(const topos_frame_output* info, uint32_t plane, uint32_t* width, uint32_t* height)
{
    if (info == NULL || width == NULL || height == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "plane geometry args NULL"); }
    if (plane >= info->plane_count) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "plane %u >= plane_count %u", plane, info->plane_count); }
    if (info->pixel_format == 3u) {
        *width = ((uint32_t)info->visible_width + 1u) / 2u;
        *height = ((uint32_t)info->visible_height + 1u) / 2u;
        return TC_OK;
    }
    const uint32_t cw = info->pixel_format == 0u ? ((uint32_t)info->visible_width + 1u) / 2u : info->visible_width;
    *width = (plane == 1u || plane == 2u) ? cw : info->visible_width;
    *height = info->visible_height;
    return TC_OK;
}

/* ============================== encode ============================== */

/* Validation and job building for one frame (reference codec.c:5730-5806 for
 * setup, :5413-5460 for per-plane qp/quantiser derivation). */
int32_t tc_prepare_encode(const topos_frame_config* cfg, const topos_frame_input* in, tcg_enc_frame* jf,
                          uint32_t* slice_count, uint8_t* qp_base)
{
    int32_t rc = tc_frame_config_validate(cfg);
    if (rc != TC_OK) { return rc; }
    if (in == NULL || (in->struct_size != 0u && in->struct_size != (uint32_t)sizeof(topos_frame_input))) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "input struct invalid");
    }
    tc_hdr h;
    tc_cfg_to_hdr(cfg, &h);
    rc = tc_hdr_geometry(&h);
    if (rc != TC_OK) { return rc; }
    const uint32_t srows = tc_cfg_slice_rows(cfg);
    uint32_t total = 0;
    rc = tc_band_plan(&h, srows, &total);
    if (rc != TC_OK) { return rc; }
    h.slices = (uint16_t)total;
    h.size = TC_HDR_SIZE;
    rc = tc_hdr_validate(&h);
    if (rc != TC_OK) { return rc; }
    for (uint32_t p = 0; p < h.planes; ++p) {
        if (in->planes[p] == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "input plane %u == NULL", p); }
        if (in->strides[p] != 0u && in->strides[p] < (size_t)h.pvw[p]) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "input stride[%u]=%zu < visible width %u", p, in->strides[p], h.pvw[p]);
        }
    }
    if (cfg->reserved[1] == 1u || cfg->reserved[2] == 1u) {
        return tc_fail(TC_ERR_NOT_IMPLEMENTED, "adaptive quantisation / RDO encode is not implemented by the GPU library");
    }
    const int v8 = h.major == 8u && h.em == 8u;
    uint32_t sb_log2 = 0u, tile_log2 = 0u;
    if (v8) {
        /* V8 segmented rANS (reference codec.c:5749-5770 granularity, 4204-4215
         * format limits): reserved[3] = segment blocks log2 (0 = 4),
         * reserved[4] = tile rows log2 (0 = 5) */
        sb_log2 = cfg->reserved[3] != 0u ? cfg->reserved[3] : 4u;
        tile_log2 = cfg->reserved[4] != 0u ? cfg->reserved[4] : 5u;
        if (sb_log2 < 3u || sb_log2 > 5u) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "v8 reserved[3] sb_log2 %u not in {3,4,5}", sb_log2);
        }
        if (tile_log2 != 0u && (tile_log2 < 4u || tile_log2 > 6u)) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "v8 reserved[4] tile_log2 %u not in {0,4,5,6}", tile_log2);
        }
        if (h.amode != 0u) { return tc_fail(TC_ERR_NOT_IMPLEMENTED, "v8 alpha pending (format-plan batch 5)"); }
        if (h.pf == 3u) { return tc_fail(TC_ERR_NOT_IMPLEMENTED, "v8 does not carry CFA (TRAW uses rans2)"); }
    } else if (!(h.major == 7u && h.em == 7u)) {
        return tc_fail(TC_ERR_NOT_IMPLEMENTED,
                       "the GPU library encodes the V7-R2 and V8 generations only (reserved[0] = 8 or 9)");
    }
    uint16_t qmL[64], qmC[64];
    if (!tc_qmatrix(h.qm, 0, qmL) || !tc_qmatrix(h.qm, 1, qmC)) {
        return tc_fail(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id %u", h.qm);
    }
    memset(jf, 0, sizeof(*jf));
    jf->planes = h.planes;
    jf->bit_depth = h.bd;
    jf->slice_rows = srows;
    jf->slices = total;
    const uint32_t refined = (h.flags & 0x8u) != 0u;
    for (uint32_t p = 0; p < h.planes; ++p) {
        tcg_enc_plane* P = &jf->plane[p];
        P->src = in->planes[p];
        P->stride = in->strides[p] != 0u ? in->strides[p] : h.pvw[p];
        P->vis_w = h.pvw[p]; P->vis_h = h.pvh[p];
        P->coded_w = h.pcw[p]; P->coded_h = h.pch[p];
        P->cols = h.bcols[p]; P->rows = h.brows[p];
        const int is_alpha = p == 3u && h.amode != 0u;
        if (is_alpha) {
            P->kind = TCG_PLANE_ALPHA;
            P->alpha_shift = h.amode == 2u ? 16u - h.abd : 0u;
            P->qdb = 64u;
        } else {
            const int chroma = h.pf != 3u && (p == 1u || p == 2u);
            const int32_t delta = chroma ? cfg->qp_delta_chroma : cfg->qp_delta_luma;
            int32_t qe = (int32_t)h.qp + delta + (h.bd >= 12u ? 2 * ((int32_t)h.bd - 10) : 0);
            if (qe < 0) { qe = 0; }
            const int32_t ceil = h.qp >= TC_QP_V15_MIN ? (int32_t)TC_QP_MAX : 63;
            if (qe > ceil) { qe = ceil; }
            P->kind = TCG_PLANE_COLOR;
            tc_quant_steps(chroma ? qmC : qmL, (uint32_t)qe, refined, P->Q);
            P->fclamp = tc_coef_clamp(h.bd);
            P->qdb = (uint32_t)(64 + qe - (int32_t)h.qp);
        }
    }
    if (v8) {
        /* the packet's slice count is the tiles of the three colour planes */
        const uint32_t tr = tile_log2 == 0u ? 0u : 1u << tile_log2;
        uint32_t tiles = 0;
        for (uint32_t p = 0; p < 3u; ++p) { tiles += (tr == 0u || h.brows[p] == 0u) ? 1u : (h.brows[p] + tr - 1u) / tr; }
        if (tiles < 3u || tiles > TC_MAX_SLICE_COUNT) {
            return tc_fail(TC_ERR_LIMIT_EXCEEDED, "v8 tile count %u out of [3,512]", tiles);
        }
        jf->v8_sb_log2 = sb_log2;
        jf->v8_tile_log2 = tile_log2;
        total = tiles;
        h.slices = (uint16_t)tiles;
    }
    tc_hdr_pack(&h, jf->header);
    *slice_count = total;
    *qp_base = h.qp;
    return TC_OK;
}

/* A V8 plane whose last segment starts past the last tile's nominal block
 * range has a segment no tile owns: the reference never codes it and its
 * post-encode self-check rejects the frame (codec.c:4289-4304). */
int tc_v8_orphans(const tcg_enc_frame* jf)
{
    if (jf->v8_sb_log2 == 0u) { return 0; }
    const uint32_t sb = 1u << jf->v8_sb_log2, tr = jf->v8_tile_log2 == 0u ? 0u : 1u << jf->v8_tile_log2;
    for (uint32_t p = 0; p < 3u; ++p) {
        const uint32_t cols = jf->plane[p].cols, rows = jf->plane[p].rows, blocks = cols * rows;
        const uint32_t S = (blocks + sb - 1u) / sb;
        const uint32_t T = (tr == 0u || rows == 0u) ? 1u : (rows + tr - 1u) / tr;
        const uint64_t fn = tr == 0u ? (uint64_t)blocks : (uint64_t)T * tr * cols;
        if (fn / sb < S) { return 1; }
    }
    return 0;
}

void tc_fill_enc_stats(topos_frame_stats* st, const tcg_enc_result* r, uint32_t slices, uint8_t qp)
{
    st->packet_size = r->packet_size;
    st->color_payload_bytes = r->color_payload;
    st->alpha_payload_bytes = r->alpha_payload;
    /* V8 (no slice headers): the frame header and the 8-byte extension */
    st->color_header_bytes = r->v8 ? TC_HDR_SIZE + 8u : TC_HDR_SIZE + TC_SH_SIZE * r->color_slices;
    st->alpha_header_bytes = TC_SH_SIZE * r->alpha_slices;
    st->slice_count = (uint16_t)slices;
    st->qp_base = qp;
    st->alpha_max_abs_error = (uint16_t)r->alpha_max_err;
}

int32_t tc_enc_result_status(int32_t rc, size_t need, size_t cap)
{
    switch (rc) {
    case TC_OK: return TC_OK;
    case TC_ERR_BUFFER_TOO_SMALL: return tc_fail(TC_ERR_BUFFER_TOO_SMALL, "out_cap %zu < %zu bytes needed", cap, need);
    case TC_ERR_LIMIT_EXCEEDED: return tc_fail(TC_ERR_LIMIT_EXCEEDED, "frame packet exceeds %u bytes", TC_MAX_PACKET);
    case TC_ERR_INVALID_ARGUMENT:
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "token domain violated (bit depth too high for this qp): raise qp or bit_depth <= 12");
    default: return rc;
    }
}

/* reference: native/src/codec/codec.c:5970-6018 (fixed-QP V7-R2 path) */
TC_EXPORT int32_t tc_frame_encode(const topos_frame_config* cfg, const topos_frame_input* input, uint8_t* out,
                                  size_t out_cap, topos_frame_stats* stats)
{
    topos_frame_stats local;
    memset(&local, 0, sizeof(local));
    if (stats == NULL) { stats = &local; }
    stats->struct_size = (uint32_t)sizeof(topos_frame_stats);
    stats->abi_version = TOPOS_CODEC_ABI_VERSION;
    if (out == NULL && out_cap != 0u) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "out == NULL with cap %zu", out_cap); }
    tcg_enc_frame jf;
    uint32_t slices = 0;
    uint8_t qp = 0;
    int32_t rc = tc_prepare_encode(cfg, input, &jf, &slices, &qp);
    if (rc != TC_OK) { return rc; }
    tcg_enc_result r;
    uint8_t* const outs[1] = {out};
    const size_t caps[1] = {out == NULL ? 0u : out_cap};
    rc = tcg_encode(&jf, 1u, outs, caps, &r);
    if (rc != TC_OK) { return rc; }
    return tc_finish_encode(&jf, &r, stats, slices, qp, out_cap);
}

/* Status and statistics of one encoded frame. V8 fills the statistics only on
 * success and reports a frame with an unowned segment after its packet was
 * written, as the reference's self-check does (codec.c:4268-4317). */
int32_t tc_finish_encode(const tcg_enc_frame* jf, tcg_enc_result* r, topos_frame_stats* stats, uint32_t slices,
                         uint8_t qp, size_t out_cap)
{
    r->v8 = jf->v8_sb_log2 != 0u;
    if (r->v8) {
        if (r->rc == TC_OK && tc_v8_orphans(jf)) {
            return tc_fail(TC_ERR_MALFORMED, "v8 self-check scan failed: a segment lies past the last tile");
        }
        if (r->rc == TC_OK) { tc_fill_enc_stats(stats, r, slices, qp); }
        return tc_enc_result_status(r->rc, r->packet_size, out_cap);
    }
    if (r->rc == TC_OK || r->rc == TC_ERR_BUFFER_TOO_SMALL) { tc_fill_enc_stats(stats, r, slices, qp); }
    return tc_enc_result_status(r->rc, r->packet_size, out_cap);
}

/* extension: many frames in one device launch sequence */
TC_EXPORT int32_t tcg_frame_encode_batch(const topos_frame_config* cfgs, const topos_frame_input* inputs, uint32_t count,
                                         uint8_t* const* outs, const size_t* out_caps, topos_frame_stats* stats,
                                         int32_t* rcs)
{
    if (count == 0u) { return TC_OK; }
    if (cfgs == NULL || inputs == NULL || outs == NULL || out_caps == NULL || rcs == NULL) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "batch arguments NULL");
    }
    if (count > TC_BATCH_MAX_FRAMES) { return tc_fail(TC_ERR_LIMIT_EXCEEDED, "batch count %u", count); }
    tcg_enc_frame* jobs = (tcg_enc_frame*)malloc(sizeof(tcg_enc_frame) * count);
    tcg_enc_result* res = (tcg_enc_result*)calloc(count, sizeof(tcg_enc_result));
    uint32_t* idx = (uint32_t*)malloc(sizeof(uint32_t) * count);
    uint32_t* nsl = (uint32_t*)calloc(count, sizeof(uint32_t));
    uint8_t* qps = (uint8_t*)calloc(count, 1);
    uint8_t** o2 = (uint8_t**)malloc(sizeof(uint8_t*) * count);
    size_t* c2 = (size_t*)malloc(sizeof(size_t) * count);
    if (!jobs || !res || !idx || !nsl || !qps || !o2 || !c2) {
        free(jobs); free(res); free(idx); free(nsl); free(qps); free(o2); free(c2);
        return tc_fail(TC_ERR_OUT_OF_MEMORY, "batch staging");
    }
    uint32_t n = 0;
    for (uint32_t i = 0; i < count; ++i) {
        if (stats != NULL) {
            memset(&stats[i], 0, sizeof(stats[i]));
            stats[i].struct_size = (uint32_t)sizeof(topos_frame_stats);
            stats[i].abi_version = TOPOS_CODEC_ABI_VERSION;
        }
        rcs[i] = tc_prepare_encode(&cfgs[i], &inputs[i], &jobs[n], &nsl[i], &qps[i]);
        if (rcs[i] == TC_OK) {
            idx[n] = i;
            o2[n] = outs[i];
            c2[n] = outs[i] == NULL ? 0u : out_caps[i];
            n++;
        }
    }
    int32_t call = TC_OK;
    if (n > 0u) { call = tcg_encode(jobs, n, o2, c2, res); }
    int32_t first = TC_OK;
    for (uint32_t k = 0; k < n && call == TC_OK; ++k) {
        const uint32_t i = idx[k];
        topos_frame_stats scratch;
        memset(&scratch, 0, sizeof(scratch));
        rcs[i] = tc_finish_encode(&jobs[k], &res[k], stats != NULL ? &stats[i] : &scratch, nsl[i], qps[i], c2[k]);
    }
    for (uint32_t i = 0; i < count; ++i) {
        if (call != TC_OK && rcs[i] == TC_OK) { rcs[i] = call; }
        if (first == TC_OK && rcs[i] != TC_OK) { first = rcs[i]; }
    }
    free(jobs); free(res); free(idx); free(nsl); free(qps); free(o2); free(c2);
    return first;
}

/* ============================== decode ============================== */

/* Generation probe + structural parse of n packets. Packets in host memory are
 * parsed in place; packets in device memory are walked on the GPU (one launch
 * for all of them) and parsed from the compact header records, so a
 * device-resident decode never copies whole packets back to the host. */
static int32_t parse_packets(const topos_batch_packet* pk, uint32_t n, tc_view* v)
{
    uint32_t ndev = 0;
    for (uint32_t i = 0; i < n; ++i) { ndev += tcg_is_device_ptr(pk[i].data) ? 1u : 0u; }
    uint8_t* rec = NULL;
    uint32_t* slot = NULL;
    if (ndev > 0u) {
        const uint8_t** ptrs = (const uint8_t**)malloc(sizeof(uint8_t*) * ndev);
        size_t* sizes = (size_t*)malloc(sizeof(size_t) * ndev);
        rec = (uint8_t*)malloc((size_t)ndev * TCG_WALK_REC);
        slot = (uint32_t*)malloc(sizeof(uint32_t) * n);
        if (ptrs == NULL || sizes == NULL || rec == NULL || slot == NULL) {
            free(ptrs); free(sizes); free(rec); free(slot);
            return tc_fail(TC_ERR_OUT_OF_MEMORY, "packet walk staging");
        }
        uint32_t k = 0;
        for (uint32_t i = 0; i < n; ++i) {
            slot[i] = UINT32_MAX;
            if (tcg_is_device_ptr(pk[i].data)) {
                ptrs[k] = pk[i].data;
                sizes[k] = pk[i].size;
                slot[i] = k++;
            }
        }
        const int32_t rc = tcg_walk_packets(ptrs, sizes, ndev, rec);
        free(ptrs);
        free(sizes);
        if (rc != TC_OK) { free(rec); free(slot); return rc; }
    }
    int32_t rc = TC_OK;
    for (uint32_t i = 0; i < n && rc == TC_OK; ++i) {
        const uint8_t* head = (slot != NULL && slot[i] != UINT32_MAX) ? rec + (size_t)slot[i] * TCG_WALK_REC : pk[i].data;
        rc = tc_probe_generation(head, pk[i].size);
        if (rc == 0) {
            rc = (slot != NULL && slot[i] != UINT32_MAX) ? tc_parse_compact(head, pk[i].size, &v[i])
                                                         : tc_parse_structure(pk[i].data, pk[i].size, &v[i]);
        }
    }
    free(rec);
    free(slot);
    return rc;
}

void tc_plan_full(tc_dec_plan* p)
{
    memset(p, 0, sizeof(*p));
    p->climit = 63u;
}

/* reference: codec.c:9366-9376 (tc_apply_decode_plan_info) */
void tc_apply_plan_info(const tc_dec_plan* plan, const tc_hdr* h, topos_frame_output* o)
{
    if (plan->tw != 0u) {  /* a resolved target, the source size included: coded = delivered */
        o->visible_width = (uint16_t)plan->tw;
        o->visible_height = (uint16_t)plan->th;
        o->coded_width = (uint16_t)plan->tw;
        o->coded_height = (uint16_t)plan->th;
    }
    if (plan->drop_alpha && o->alpha_mode != 0u && o->plane_count >= 4u) {
        o->plane_count = 3u;
        o->alpha_mode = 0u;
        o->alpha_bit_depth = 0u;
    }
    (void)h;
}

static int32_t build_decode(const tc_view* v, const uint8_t* data, uint16_t* const* planes_out, const size_t* strides,
                            const tc_dec_plan* plan, tcg_dec_frame* jf, tcg_dec_slice* sl, topos_frame_output* o)
{
    const tc_hdr* h = &v->h;
    memset(jf, 0, sizeof(*jf));
    const uint32_t np = (plan->drop_alpha && h->amode != 0u && h->planes >= 4u) ? 3u : h->planes;
    for (uint32_t p = 0; p < np; ++p) {
        if (planes_out[p] == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "planes_out[%u] == NULL", p); }
        uint32_t dw = h->pvw[p], dh = h->pvh[p];
        if (plan->scaled) {
            const int c422 = h->pf == 0u && (p == 1u || p == 2u);
            dw = c422 ? (plan->tw + 1u) / 2u : plan->tw;
            dh = plan->th;
        }
        const size_t s = strides != NULL ? strides[p] : 0u;
        if (s != 0u && s < (size_t)dw) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "plane %u stride %zu < visible width %u", p, s, dw);
        }
        jf->dst[p] = planes_out[p];
        jf->dst_stride[p] = s;
        jf->dst_w[p] = dw;
        jf->dst_h[p] = dh;
        jf->vis_w[p] = h->pvw[p]; jf->vis_h[p] = h->pvh[p]; jf->coded_w[p] = h->pcw[p];
        jf->cols[p] = h->bcols[p]; jf->rows[p] = h->brows[p];
        const int chroma = h->pf != 3u && (p == 1u || p == 2u);
        if (!tc_qmatrix(h->qm, chroma, jf->qm[p])) { return tc_fail(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id %u", h->qm); }
    }
    jf->packet = data;
    jf->size = h->size;
    jf->planes = np;
    jf->climit = plan->climit;
    jf->scaled = plan->scaled;
    /* deblocking grid of the delivered planes (reference codec.c:8649-8660) */
    jf->db_unit = (h->flags & 0x4u) == 0u ? 0u
                  : !plan->scaled ? 8u
                  : (plan->tw * 2u == h->vw && plan->th * 2u == h->vh) ? 4u : 0u;
    jf->bit_depth = h->bd;
    jf->alpha_mode = h->amode;
    jf->alpha_shift = h->amode == 2u ? 16u - h->abd : 0u;
    jf->refined = (h->flags & 0x8u) != 0u;
    jf->deblock = (h->flags & 0x4u) != 0u;
    jf->qp_base = h->qp;
    jf->slices = h->slices;
    for (uint32_t i = 0; i < h->slices; ++i) {
        const tc_shdr* s = &v->s[i];
        sl[i].off = v->off[i];
        sl[i].size = s->size;
        sl[i].crc = s->crc;
        sl[i].plane = s->plane;
        sl[i].y0 = s->y0;
        sl[i].bh = s->bh;
        sl[i].qp = (uint16_t)((int32_t)h->qp + (int32_t)s->qdb - 64);
        sl[i].k1 = s->k1;
        sl[i].k2 = s->k2;
    }
    jf->slice = sl;
    jf->slice_status = o->slice_status;
    return TC_OK;
}

static int32_t finish_frame(const tc_hdr* h, topos_frame_output* o)
{
    uint32_t concealed = 0;
    for (uint32_t i = 0; i < h->slices; ++i) { concealed += o->slice_status[i] != 0u; }
    o->concealed_slices = (uint16_t)concealed;
    if (concealed != 0u) {
        tc_fail(TC_WARN_CONCEALED, "%u of %u slices concealed", concealed, h->slices);
        return TC_WARN_CONCEALED;
    }
    return TC_OK;
}

/* version_major of a packet in host or device memory (-1: no TPIC header) */
int tc_packet_major(const uint8_t* data, size_t size)
{
    uint8_t head[8] = {0};
    if (data == NULL || size < TC_HDR_SIZE) { return -1; }
    if (tcg_is_device_ptr(data)) {
        if (tcg_read_device(head, data, 8u) != TC_OK) { return -1; }
    } else {
        memcpy(head, data, 8u);
    }
    return memcmp(head, "TPIC", 4u) == 0 ? (int)head[6] : -1;
}

/* reference: native/src/codec/codec.c:9005-9098 */
TC_EXPORT int32_t tc_frame_decode(const uint8_t* data, size_t size, uint16_t* const planes_out[TC_FRAME_MAX_PLANES],
                                  const size_t strides[TC_FRAME_MAX_PLANES], topos_frame_output* o)
{
    if (o == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "out_info == NULL"); }
    memset(o, 0, sizeof(*o));
    o->struct_size = (uint32_t)sizeof(topos_frame_output);
    o->abi_version = TOPOS_CODEC_ABI_VERSION;
    if (data == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "data == NULL"); }
    /* V8 packets take their own decoder (reference codec.c:9039-9049) */
    if (tc_packet_major(data, size) == 8) { return tc_v8_frame_decode(data, size, planes_out, strides, o); }
    tc_view* v = (tc_view*)malloc(sizeof(tc_view));
    if (v == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "decode view"); }
    const topos_batch_packet one = {data, size};
    int32_t rc = parse_packets(&one, 1u, v);
    if (rc != TC_OK) { free(v); return rc; }
    tc_fill_info(&v->h, o);
    if (planes_out == NULL) { free(v); return TC_OK; }
    if (v->h.major == 7u && v->h.em == 8u && v->h.ftype != 0u) {
        free(v);
        return tc_fail(TC_ERR_STATE, "v7r3 P-frame decode requires a GOP context (stateless entry is I-only)");
    }
    if (!(v->h.major == 7u && (v->h.em == 7u || v->h.em == 8u))) {
        free(v);
        return tc_fail(TC_ERR_NOT_IMPLEMENTED, "the GPU library decodes V7-R2 intra packets only");
    }
    tcg_dec_frame jf;
    tcg_dec_slice sl[TC_MAX_SLICE_COUNT];
    tc_dec_plan full;
    tc_plan_full(&full);
    rc = build_decode(v, data, planes_out, strides, &full, &jf, sl, o);
    if (rc == TC_OK) { rc = tcg_decode(&jf, 1u); }
    if (rc == TC_OK) { rc = finish_frame(&v->h, o); }
    free(v);
    return rc;
}

/* Allocation-free form of tc_frame_decode_batch's query mode (no reference
 * counterpart). Every buffer is on the stack or in the device library's static
 * scratch; packets in device memory are walked with the static-scratch walk
 * and parsed from their records one at a time, each record copied once. Like
 * the batch query, infos is left untouched when any packet fails. */
TC_EXPORT int32_t tcg_frame_query_batch_noalloc(const topos_batch_packet* packets, uint32_t count,
                                                topos_frame_output* infos)
{
    if (count == 0u) { return TC_OK; }
    if (count > TCG_NOALLOC_MAX_PACKETS) {
        return tc_fail(TC_ERR_LIMIT_EXCEEDED, "allocation-free query: count %u > %u", count,
                       (unsigned)TCG_NOALLOC_MAX_PACKETS);
    }
    if (infos == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "infos == NULL"); }
    if (packets == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "batch packets == NULL"); }
    const uint8_t* dptrs[TCG_NOALLOC_MAX_PACKETS];
    size_t dsizes[TCG_NOALLOC_MAX_PACKETS];
    uint32_t slot[TCG_NOALLOC_MAX_PACKETS];
    uint32_t ndev = 0;
    for (uint32_t i = 0; i < count; ++i) {
        if (packets[i].data == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "packets[%u].data == NULL", i); }
        slot[i] = UINT32_MAX;
        if (tcg_is_device_ptr(packets[i].data)) {
            dptrs[ndev] = packets[i].data;
            dsizes[ndev] = packets[i].size;
            slot[i] = ndev++;
        }
    }
    if (ndev > 0u) {
        const int32_t rc = tcg_walk_packets_noalloc(dptrs, dsizes, ndev);
        if (rc != TC_OK) { return rc; }
    }
    /* each record is copied and parsed once; only the frame headers are kept
     * until every packet has parsed, so infos stays untouched on a failure */
    uint8_t rec[TCG_WALK_REC];
    tc_view v;
    tc_hdr hdrs[TCG_NOALLOC_MAX_PACKETS];
    for (uint32_t i = 0; i < count; ++i) {
        const int dev = slot[i] != UINT32_MAX;
        if (dev) {
            const int32_t rc = tcg_walk_record_noalloc(slot[i], rec);
            if (rc != TC_OK) { return rc; }
        }
        const uint8_t* head = dev ? rec : packets[i].data;
        int32_t rc = tc_probe_generation(head, packets[i].size);
        if (rc == 0) {
            rc = dev ? tc_parse_compact(head, packets[i].size, &v) : tc_parse_structure(packets[i].data, packets[i].size, &v);
        }
        if (rc != TC_OK) { return rc; }
        hdrs[i] = v.h;
    }
    for (uint32_t i = 0; i < count; ++i) {
        topos_frame_output* o = &infos[i];
        memset(o, 0, sizeof(*o));
        o->struct_size = (uint32_t)sizeof(topos_frame_output);
        o->abi_version = TOPOS_CODEC_ABI_VERSION;
        tc_fill_info(&hdrs[i], o);
    }
    return TC_OK;
}

/* reference: native/src/codec/codec.c:9639-9789 (tc_frame_decode_batch_mode),
 * decoder_ctx.c:652-760 (its plan-resolving form) */
int32_t tc_decode_batch_mode(const topos_batch_packet* packets, uint32_t count, uint16_t* const* planes_out,
                             const size_t* strides, topos_frame_output* infos, tc_plan_fn fn, const void* ctx)
{
    if (count == 0u) { return TC_OK; }
    if (count > TC_BATCH_MAX_FRAMES) { return tc_fail(TC_ERR_LIMIT_EXCEEDED, "batch count %u > %u", count, TC_BATCH_MAX_FRAMES); }
    if (infos == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "infos == NULL"); }
    if (packets == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "batch packets == NULL"); }
    for (uint32_t i = 0; i < count; ++i) {
        if (packets[i].data == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "packets[%u].data == NULL", i); }
    }
    tc_view* v = (tc_view*)malloc(sizeof(tc_view) * count);
    if (v == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "decode batch context"); }
    {
        const int32_t rc = parse_packets(packets, count, v);
        if (rc != TC_OK) { free(v); return rc; }
    }
    int32_t* frc = (int32_t*)calloc(count, sizeof(int32_t));
    tc_dec_plan* plans = (tc_dec_plan*)calloc(count, sizeof(tc_dec_plan));
    tcg_dec_frame* jf = planes_out != NULL ? (tcg_dec_frame*)calloc(count, sizeof(tcg_dec_frame)) : NULL;
    tcg_dec_slice* sl = planes_out != NULL
        ? (tcg_dec_slice*)calloc((size_t)count * TC_MAX_SLICE_COUNT, sizeof(tcg_dec_slice)) : NULL;
    if (frc == NULL || plans == NULL || (planes_out != NULL && (jf == NULL || sl == NULL))) {
        free(v); free(frc); free(plans); free(jf); free(sl);
        return tc_fail(TC_ERR_OUT_OF_MEMORY, "decode batch staging");
    }
    int32_t call = TC_OK;
    for (uint32_t i = 0; i < count && call == TC_OK; ++i) {
        topos_frame_output* o = &infos[i];
        memset(o, 0, sizeof(*o));
        o->struct_size = (uint32_t)sizeof(topos_frame_output);
        o->abi_version = TOPOS_CODEC_ABI_VERSION;
        tc_fill_info(&v[i].h, o);
        if (planes_out != NULL && v[i].h.major == 7u && v[i].h.em == 8u && v[i].h.ftype != 0u) {
            call = tc_fail(TC_ERR_STATE, "v7r3 P-frame decode requires a GOP context (stateless entry is I-only)");
            break;
        }
        tc_plan_full(&plans[i]);
        if (fn != NULL) {
            const int32_t prc = fn(ctx, &v[i].h, &plans[i]);
            if (prc != TC_OK) {
                if (planes_out == NULL) { call = prc; break; }
                frc[i] = prc;
                continue;
            }
        }
        tc_apply_plan_info(&plans[i], &v[i].h, o);
        if (planes_out == NULL) { continue; }
        for (uint32_t p = 0; p < o->plane_count; ++p) {
            if (planes_out[(size_t)i * 4u + p] == NULL) {
                frc[i] = tc_fail(TC_ERR_INVALID_ARGUMENT, "frame %u planes_out[%u] == NULL", i, p);
                break;
            }
        }
    }
    if (call != TC_OK || planes_out == NULL) {
        free(v); free(frc); free(plans); free(jf); free(sl);
        return call;
    }
    for (uint32_t i = 0; i < count; ++i) {
        jf[i].skip = 1;
        if (frc[i] != TC_OK) { continue; }
        if (!(v[i].h.major == 7u && (v[i].h.em == 7u || v[i].h.em == 8u))) {
            frc[i] = tc_fail(TC_ERR_NOT_IMPLEMENTED, "the GPU library decodes V7-R2 intra packets only");
            continue;
        }
        frc[i] = build_decode(&v[i], packets[i].data, planes_out + (size_t)i * 4u,
                              strides != NULL ? strides + (size_t)i * 4u : NULL, &plans[i], &jf[i],
                              sl + (size_t)i * TC_MAX_SLICE_COUNT, &infos[i]);
        jf[i].skip = frc[i] != TC_OK;
    }
    call = tcg_decode(jf, count);
    int32_t first = TC_OK;
    for (uint32_t i = 0; i < count; ++i) {
        if (frc[i] == TC_OK) { frc[i] = call != TC_OK ? call : finish_frame(&v[i].h, &infos[i]); }
        if (first == TC_OK) { first = frc[i]; }
    }
    free(v); free(frc); free(plans); free(jf); free(sl);
    return first;
}

/* reference: native/src/codec/codec.c:9791-9805 */
TC_EXPORT int32_t tc_frame_decode_batch(const topos_batch_packet* packets, uint32_t count, uint16_t* const* planes_out,
                                        const size_t* strides, topos_frame_output* infos)
{
    return tc_decode_batch_mode(packets, count, planes_out, strides, infos, NULL, NULL);
}

/* ============================== device control ============================== */

TC_EXPORT int32_t tcg_device_init(int32_t device) { return tcg_init(device); }
TC_EXPORT void tcg_device_release(void) { tcg_shutdown(); }

TC_EXPORT void tcg_release_idle_memory(void) { tcg_trim_idle(); }
TC_EXPORT uint64_t tcg_kernel_launches(void) { return tcg_launch_count(); }
TC_EXPORT double tcg_last_device_ms(void) { return tcg_last_ms(); }
TC_EXPORT uint32_t tcg_pipeline_plan(int32_t decode, const uint64_t* frame_bytes, uint32_t count, uint32_t* starts)
{
    return tcg_pipeline_chunks(decode, frame_bytes, count, starts);
}
TC_EXPORT void tcg_profile_enable(int32_t on) { tcg_prof_enable(on); }
TC_EXPORT void tcg_profile_reset(void) { tcg_prof_reset(); }
TC_EXPORT int32_t tcg_profile_read(uint32_t id, const char** name, double* ms, uint64_t* launches)
{
    return tcg_prof_read(id, name, ms, launches);
}
