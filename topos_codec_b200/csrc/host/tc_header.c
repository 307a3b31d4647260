/* tc_header.c - frame/slice header rules, slice planning and packet structure.
 *
 * The field rules, their order and their status codes follow the reference
 * exactly because callers observe them: header validation
 * (native/src/bitstream/frame_header.c:99-535), geometry (:541-588), header
 * pack/decode (:590-631, :703-781), config -> header mapping
 * (native/src/codec/codec.c:280-397), slice planning (:405-424), structural
 * parse (native/src/bitstream/packet.c:13-67) and tiling validation
 * (native/src/bitstream/slice_map.c:48-143).
 */
#include <string.h>

#include "tc_internal.h"

static void be16(uint8_t* p, uint32_t v) { p[0] = (uint8_t)(v >> 8); p[1] = (uint8_t)v; }
static void be32(uint8_t* p, uint32_t v)
{
    p[0] = (uint8_t)(v >> 24); p[1] = (uint8_t)(v >> 16); p[2] = (uint8_t)(v >> 8); p[3] = (uint8_t)v;
}
static uint32_t ld16(const uint8_t* p) { return ((uint32_t)p[0] << 8) | p[1]; }
static uint32_t ld32(const uint8_t* p)
{
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

static int32_t vf(int32_t code, const char* field, unsigned long long v)
{
    return tc_fail(code, "frame header field %s = %llu rejected", field, v);
}

static int32_t vretire(unsigned major)
{
    return tc_fail(TC_ERR_UNSUPPORTED_VERSION,
                   "generation %u retired; archived streams are not decodable", major);
}

int32_t tc_hdr_validate(const tc_hdr* h)
{
    const unsigned M = h->major;
    if (M >= 2u && M <= 9u) {
        if (M >= 3u && M <= 6u) { return vretire(M); }
        if (M == 2u && h->em == 0u) { return vretire(2u); }
        if (M == 7u && h->em == 6u) { return vretire(7u); }
        if (h->minor != 0u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "v2 version_minor", h->minor); }
        if (M == 7u) {
            if (!((h->em == 6u || h->em == 7u || h->em == 8u) && h->cb == 0u && h->cm == 0u)) {
                return vf(TC_ERR_UNSUPPORTED_VERSION, "v7 rans entropy fields", h->em);
            }
        } else if (M == 8u || M == 9u) {
            if (!(h->em == M && h->cb == 0u && h->cm == 0u)) {
                return vf(TC_ERR_UNSUPPORTED_VERSION, "v8/v9 entropy fields", h->em);
            }
        } else if (h->em > 1u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "entropy_mode", h->em);
        }
        if (M == 2u && (h->em == 0u ? h->cb != 0u : h->cb != 1u)) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "codebook_version", h->cb);
        }
        if (M == 2u && h->cm != 0u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "coding_mode", h->cm); }
        if ((h->flags & ~0x0003u) != 0u) {
            if ((h->flags & ~0x000Fu) != 0u) { return vf(TC_ERR_MALFORMED, "v2 flags(reserved bits)", h->flags); }
            if ((h->flags & 0x000Cu) != 0u &&
                !(M == 7u && h->em == 7u && h->ftype == 0u && h->profile == 3u && h->bd == 10u)) {
                return vf(TC_ERR_UNSUPPORTED_VERSION, "flags r4/r5 domain", h->flags);
            }
        }
        if ((h->flags & 0x0002u) != 0u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "tile_layout(V2.0)", h->flags); }
        if (M == 9u || (M == 7u && h->em == 8u)) {
            if (h->ftype > 1u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "v9 frame_type", h->ftype); }
            if (h->ftype == 0u && h->refd != 0u) { return vf(TC_ERR_MALFORMED, "v9 I ref_distance(!=0)", h->refd); }
            if (h->ftype == 1u && h->refd != 1u) { return vf(TC_ERR_MALFORMED, "v9 P ref_distance(!=1)", h->refd); }
        } else if (h->ftype != 0u || h->gop != 0u || h->refd != 0u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "frame_type/gop/ref(V2.1)", h->ftype);
        }
    } else if (M != 1u) {
        return vf(TC_ERR_UNSUPPORTED_VERSION, "version_major", M);
    } else {
        if (h->em != 0u || h->cb != 0u || h->cm != 0u) { return vf(TC_ERR_MALFORMED, "v1 entropy fields(!=0)", h->em); }
        if ((h->flags & ~0x0001u) != 0u) { return vf(TC_ERR_MALFORMED, "flags(reserved bits)", h->flags); }
        if (h->ftype != 0u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "frame_type(V2.1)", h->ftype); }
        if (h->gop != 0u) { return vf(TC_ERR_MALFORMED, "gop_id(reserved)", h->gop); }
        if (h->refd != 0u) { return vf(TC_ERR_MALFORMED, "ref_distance(reserved)", h->refd); }
    }
    if (h->profile < 1u || h->profile > 7u) { return vf(TC_ERR_UNSUPPORTED_PROFILE, "profile", h->profile); }
    if (h->profile == 7u) {
        if (h->pf != 3u) { return vf(TC_ERR_MALFORMED, "profile(TRAW requires CFA pf=3)", h->pf); }
        if (h->bd != 12u && h->bd != 16u) { return vf(TC_ERR_MALFORMED, "profile(TRAW requires 12/16-bit)", h->bd); }
        if (h->amode != 0u) { return vf(TC_ERR_MALFORMED, "profile(TRAW alpha unsupported)", h->amode); }
        if (h->qm != 0u) { return vf(TC_ERR_MALFORMED, "profile(TRAW frozen qm0)", h->qm); }
        if (h->xfer != (h->bd == 12u ? TC_TRAW_LOG0 : 8u)) {
            return vf(TC_ERR_MALFORMED, "profile(TRAW transfer mismatch for bit depth)", h->xfer);
        }
    } else {
        if (h->profile != 3u && h->profile != 5u && h->profile != 6u) {
            return vf(TC_ERR_UNSUPPORTED_PROFILE, "profile(not 3/5/6)", h->profile);
        }
        if (h->pf == 3u) { return vf(TC_ERR_MALFORMED, "pixel_format(CFA requires TRAW profile 7)", h->pf); }
    }
    if (h->profile == 5u || h->profile == 6u) {
        if (h->pf == 0u) { return vf(TC_ERR_MALFORMED, "profile/format(Pro444|Extreme requires 4:4:4)", h->pf); }
        if (h->profile == 6u && h->bd != 12u) { return vf(TC_ERR_MALFORMED, "profile/format(Extreme requires 12-bit)", h->bd); }
    }
    if (h->pf > 3u) { return vf(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "pixel_format", h->pf); }
    if (h->bd != 10u && h->bd != 12u && h->bd != 16u) { return vf(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "bit_depth", h->bd); }
    if (M == 1u) {
        if (h->minor > 7u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "version_minor", h->minor); }
        if (h->minor == 0u && (h->bd != 10u || h->pf != 0u)) { return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.2 extended enum in minor 0", h->bd); }
        if (h->minor == 1u && h->pf != 0u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.3 extended enum in minor 1", h->pf); }
        if (h->minor == 2u && h->pf > 1u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.4 extended enum in minor 2", h->pf); }
        if (h->minor < 5u && (h->pf == 3u || h->profile == 7u)) { return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.6 extended enum in minor<5", h->pf); }
        if (h->minor < 6u && h->bd == 16u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.7 extended enum in minor<6", h->bd); }
    }
    if (h->amode > 2u) { return vf(TC_ERR_MALFORMED, "alpha_mode", h->amode); }
    if (h->amode == 0u) {
        if (h->abd != 0u) { return vf(TC_ERR_MALFORMED, "alpha_bit_depth(!=0 w/o alpha)", h->abd); }
    } else if (h->amode == 1u) {
        if (h->abd != 16u) { return vf(TC_ERR_MALFORMED, "alpha_bit_depth(!=16 lossless)", h->abd); }
    } else if (h->abd != 8u && h->abd != 10u && h->abd != 12u) {
        return vf(TC_ERR_MALFORMED, "alpha_bit_depth(near-lossless)", h->abd);
    }
    if (h->cw == 0u || h->ch == 0u || (h->cw % 8u) != 0u || (h->ch % 8u) != 0u ||
        h->cw > TC_MAX_DIM || h->ch > TC_MAX_DIM) {
        return vf(TC_ERR_LIMIT_EXCEEDED, "coded_w/h(16384,%8)", h->cw);
    }
    if (h->vw == 0u || h->vh == 0u) { return vf(TC_ERR_MALFORMED, "visible_w/h(>=1)", h->vw); }
    if (h->vw > h->cw || h->vh > h->ch) { return vf(TC_ERR_LIMIT_EXCEEDED, "visible>coded", h->vw); }
    const uint8_t ep = h->pf == 3u ? 4u : (uint8_t)(3u + (h->amode != 0u ? 1u : 0u));
    if (h->planes != ep) { return vf(TC_ERR_MALFORMED, "plane_count", h->planes); }
    if (h->qm > 4u) { return vf(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id", h->qm); }
    if (h->qm == 2u && !(h->pf == 2u && h->bd == 12u && (h->profile == 5u || h->profile == 6u))) {
        return vf(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id=2 domain", h->qm);
    }
    if ((h->qm == 3u || h->qm == 4u) && !(h->pf == 0u && h->bd == 10u && h->profile == 3u)) {
        return vf(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id=3/4 domain", h->qm);
    }
    if (h->qp > TC_QP_MAX) { return vf(TC_ERR_MALFORMED, "qp_base", h->qp); }
    if (h->qp >= TC_QP_V15_MIN && !((M == 1u && h->minor >= 4u) || M >= 2u)) {
        return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.5 qp>=64 in minor<4", h->qp);
    }
    if (h->slices == 0u) { return vf(TC_ERR_MALFORMED, "slice_count(>=1)", h->slices); }
    if (h->slices > TC_MAX_SLICE_COUNT) { return vf(TC_ERR_LIMIT_EXCEEDED, "slice_count(<=512)", h->slices); }
    if (h->slices < h->planes) { return vf(TC_ERR_MALFORMED, "slice_count(<plane_count)", h->slices); }
    if (h->range > 1u) { return vf(TC_ERR_MALFORMED, "color_range", h->range); }
    if (h->siting > 2u) { return vf(TC_ERR_MALFORMED, "chroma_siting", h->siting); }
    if ((h->pf == 2u || h->pf == 3u) && h->siting != 0u) { return vf(TC_ERR_MALFORMED, "chroma_siting(GBR|CFA)", h->siting); }
    switch (h->prim) {
    case 1: case 6: case 9: case 12: break;
    default: return vf(TC_ERR_MALFORMED, "color_primaries(tag)", h->prim);
    }
    switch (h->xfer) {
    case 1: case 8: case 16: case 18: case TC_TRAW_LOG0: break;
    case 13:
        if (M == 1u && h->minor < 7u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.8 sRGB transfer in minor<7", h->minor); }
        break;
    default: return vf(TC_ERR_MALFORMED, "color_transfer(tag)", h->xfer);
    }
    if (h->profile == 7u) {
        if (h->xfer != (h->bd == 16u ? 8u : TC_TRAW_LOG0)) { return vf(TC_ERR_MALFORMED, "color_transfer(profile7 pair)", h->xfer); }
    } else if (h->xfer == TC_TRAW_LOG0) {
        return vf(TC_ERR_MALFORMED, "color_transfer(TRAW_LOG0 is profile-7 private)", h->xfer);
    }
    if (h->pf == 2u || h->pf == 3u) {
        if (h->matrix != 0u) { return vf(TC_ERR_MALFORMED, "color_matrix(!=0 identity for GBR)", h->matrix); }
    } else {
        switch (h->matrix) {
        case 1: case 5: case 9: break;
        default: return vf(TC_ERR_MALFORMED, "color_matrix(tag)", h->matrix);
        }
    }
    if ((h->sarn == 0u) != (h->sard == 0u)) { return vf(TC_ERR_MALFORMED, "sar(0 iff 0)", h->sarn); }
    if (h->size == 0u || h->size > TC_MAX_PACKET) { return vf(TC_ERR_LIMIT_EXCEEDED, "frame_packet_size(<=256MiB)", h->size); }
    return TC_OK;
}

int32_t tc_hdr_geometry(tc_hdr* h)
{
    if (h->pf == 3u) {
        const uint32_t w = ((uint32_t)h->vw + 1u) / 2u, hh = ((uint32_t)h->vh + 1u) / 2u;
        const uint32_t cw = (w + 7u) / 8u * 8u, ch = (hh + 7u) / 8u * 8u;
        for (int p = 0; p < 4; ++p) {
            h->pcw[p] = (uint16_t)cw; h->pch[p] = (uint16_t)ch;
            h->pvw[p] = (uint16_t)w; h->pvh[p] = (uint16_t)hh;
            h->bcols[p] = (uint16_t)(cw / 8u); h->brows[p] = (uint16_t)(ch / 8u);
        }
        if (cw > TC_MAX_DIM || ch > TC_MAX_DIM) { return tc_fail(TC_ERR_LIMIT_EXCEEDED, "cfa plane coded dim exceeds 16384"); }
        return TC_OK;
    }
    const uint32_t cvw = h->pf == 0u ? ((uint32_t)h->vw + 1u) / 2u : h->vw;
    const uint32_t ccw = h->pf == 0u ? (cvw + 7u) / 8u * 8u : h->cw;
    for (int p = 0; p < 4; ++p) {
        const int c = p == 1 || p == 2;
        h->pcw[p] = (uint16_t)(c ? ccw : h->cw);
        h->pch[p] = h->ch;
        h->pvw[p] = (uint16_t)(c ? cvw : h->vw);
        h->pvh[p] = h->vh;
        h->bcols[p] = (uint16_t)(h->pcw[p] / 8u);
        h->brows[p] = (uint16_t)(h->pch[p] / 8u);
    }
    if (h->pcw[1] > TC_MAX_DIM || h->pch[1] > TC_MAX_DIM) { return tc_fail(TC_ERR_LIMIT_EXCEEDED, "chroma coded dim exceeds 16384"); }
    return TC_OK;
}

void tc_hdr_pack(const tc_hdr* h, uint8_t o[TC_HDR_SIZE])
{
    o[0] = 'T'; o[1] = 'P'; o[2] = 'I'; o[3] = 'C';
    be16(o + 4, TC_HDR_SIZE);
    o[6] = h->major; o[7] = h->minor;
    be16(o + 8, h->flags);
    o[10] = h->profile; o[11] = h->pf; o[12] = h->bd; o[13] = h->amode; o[14] = h->abd;
    o[15] = h->ftype; be16(o + 16, h->gop); o[18] = h->refd;
    be16(o + 19, h->cw); be16(o + 21, h->ch); be16(o + 23, h->vw); be16(o + 25, h->vh);
    o[27] = h->planes; o[28] = h->qm; o[29] = h->qp;
    be16(o + 30, h->slices);
    o[32] = h->range; o[33] = h->prim; o[34] = h->xfer; o[35] = h->matrix; o[36] = h->siting;
    be16(o + 37, h->sarn); be16(o + 39, h->sard);
    be32(o + 41, h->size);
    o[45] = h->em; o[46] = h->cb; o[47] = h->cm; o[48] = 0u;
    be32(o + 49, tc_crc32(o, 49u));
}

int32_t tc_hdr_decode(const uint8_t* d, size_t n, tc_hdr* h);

static int32_t hdr_decode(const uint8_t* d, size_t n, tc_hdr* h)
{
    if (n < TC_HDR_SIZE) { return tc_fail(TC_ERR_TRUNCATED, "frame header needs 53 bytes, got %zu", n); }
    if (memcmp(d, "TPIC", 4u) != 0) { return tc_fail(TC_ERR_MALFORMED, "magic mismatch (not TPIC)"); }
    const uint32_t crc = tc_crc32(d, 49u);
    if (ld32(d + 49) != crc) { return tc_fail(TC_ERR_CHECKSUM_MISMATCH, "frame header crc32 %08x != %08x", ld32(d + 49), crc); }
    memset(h, 0, sizeof(*h));
    if (ld16(d + 4) != TC_HDR_SIZE) { return vf(TC_ERR_MALFORMED, "header_size(!=53)", ld16(d + 4)); }
    const uint8_t M = d[6];
    if (M >= 3u && M <= 6u) { return vretire(M); }
    if (M < 1u || M > 9u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "version_major", M); }
    h->major = M; h->minor = d[7];
    h->flags = (uint16_t)ld16(d + 8);
    h->profile = d[10]; h->pf = d[11]; h->bd = d[12]; h->amode = d[13]; h->abd = d[14];
    h->ftype = d[15]; h->gop = (uint16_t)ld16(d + 16); h->refd = d[18];
    h->cw = (uint16_t)ld16(d + 19); h->ch = (uint16_t)ld16(d + 21);
    h->vw = (uint16_t)ld16(d + 23); h->vh = (uint16_t)ld16(d + 25);
    h->planes = d[27]; h->qm = d[28]; h->qp = d[29];
    h->slices = (uint16_t)ld16(d + 30);
    h->range = d[32]; h->prim = d[33]; h->xfer = d[34]; h->matrix = d[35]; h->siting = d[36];
    h->sarn = (uint16_t)ld16(d + 37); h->sard = (uint16_t)ld16(d + 39);
    h->size = ld32(d + 41);
    if (M == 1u) {
        if (ld32(d + 45) != 0u) { return vf(TC_ERR_MALFORMED, "reserved0(!=0)", ld32(d + 45)); }
    } else {
        h->em = d[45]; h->cb = d[46]; h->cm = d[47];
        if (d[48] != 0u) { return vf(TC_ERR_MALFORMED, "reserved_v2_0(!=0)", d[48]); }
    }
    int32_t rc = tc_hdr_validate(h);
    if (rc != TC_OK) { return rc; }
    return tc_hdr_geometry(h);
}

static void select_minor(tc_hdr* h)
{
    if (h->major >= 2u) { h->minor = 0u; return; }
    h->minor = h->bd == 16u ? 6u : h->pf == 3u ? 5u : h->pf == 2u ? 3u : h->pf == 1u ? 2u
               : h->bd != 10u ? 1u : 0u;
    if (h->qp >= TC_QP_V15_MIN && h->minor < 4u) { h->minor = 4u; }
    if (h->xfer == 13u && h->minor < 7u) { h->minor = 7u; }
}

void tc_cfg_to_hdr(const topos_frame_config* c, tc_hdr* h)
{
    memset(h, 0, sizeof(*h));
    h->flags = c->alpha_premultiplied != 0u ? 1u : 0u;
    if ((c->reserved[0] & 0xFFu) == 8u && c->reserved[5] != 0u) {
        h->flags = (uint16_t)(h->flags | ((c->reserved[5] & 1u) ? 0x4u : 0u) | ((c->reserved[5] & 2u) ? 0x8u : 0u));
    }
    h->profile = c->profile != 0u ? c->profile : (c->pixel_format == 3u ? 7u : 3u);
    h->pf = c->pixel_format;
    h->bd = c->bit_depth != 0u ? c->bit_depth : 10u;
    h->matrix = c->color_matrix != 0u ? c->color_matrix : (h->pf == 2u || h->pf == 3u ? 0u : 1u);
    h->qp = c->qp_base;
    select_minor(h);
    h->amode = c->alpha_mode;
    h->abd = c->alpha_bit_depth;
    h->cw = (uint16_t)((c->visible_width + 7u) / 8u * 8u);
    h->ch = (uint16_t)((c->visible_height + 7u) / 8u * 8u);
    h->vw = c->visible_width;
    h->vh = c->visible_height;
    h->planes = (uint8_t)(c->pixel_format == 3u ? 4u : 3u + (c->alpha_mode != 0u ? 1u : 0u));
    h->qm = c->qmatrix_id;
    h->range = c->color_range;
    h->prim = c->color_primaries != 0u ? c->color_primaries : 1u;
    h->xfer = c->color_transfer != 0u ? c->color_transfer
              : (c->pixel_format == 3u ? (c->bit_depth == 16u ? 8u : TC_TRAW_LOG0) : 13u);
    h->siting = c->chroma_siting;
    select_minor(h);
    h->sarn = c->sar_num;
    h->sard = c->sar_den;
    const uint8_t em = (uint8_t)(c->reserved[0] & 0xFFu);
    if (em == 8u) { h->major = 7u; h->em = 7u; }
    else if (em == 9u) { h->major = 8u; h->em = 8u; }
    else if (em == 10u || em == 11u) {
        h->major = em == 10u ? 9u : 7u;
        h->em = em == 10u ? 9u : 8u;
        h->ftype = (uint8_t)c->reserved[3];
        h->gop = (uint16_t)c->reserved[4];
        h->refd = (uint8_t)c->reserved[5];
    } else if (em == 1u) { h->major = 2u; h->em = 1u; h->cb = 1u; }
    else { h->major = 1u; }
    if (h->major >= 2u) { select_minor(h); }
}

uint32_t tc_cfg_slice_rows(const topos_frame_config* c)
{
    return c->slice_rows != 0u ? c->slice_rows : TC_FRAME_DEFAULT_SLICE_ROWS;
}

int32_t tc_band_plan(const tc_hdr* h, uint32_t rows_per, uint32_t* total)
{
    uint64_t t = 0;
    for (uint32_t p = 0; p < h->planes; ++p) {
        const uint64_t b = ((uint64_t)h->brows[p] + rows_per - 1u) / rows_per;
        t += b == 0u ? 1u : b;
    }
    if (t > TC_MAX_SLICE_COUNT) {
        return tc_fail(TC_ERR_LIMIT_EXCEEDED, "slice_rows %u yields %llu slices > 512", rows_per, (unsigned long long)t);
    }
    if (total != NULL) { *total = (uint32_t)t; }
    return TC_OK;
}

int32_t tc_hdr_decode(const uint8_t* d, size_t n, tc_hdr* h) { return hdr_decode(d, n, h); }

/* V8 (major 8) is not intercepted: the single-frame decode routes it to the V8
 * decoder first, and the V7 scanner rejects it elsewhere (packet.c:19-26). */
int32_t tc_probe_generation(const uint8_t* d, size_t n)
{
    if (n >= TC_HDR_SIZE + 8u && memcmp(d, "TPIC", 4u) == 0 && d[6] == 7u &&
        memcmp(d + TC_HDR_SIZE, "TPLD", 4u) == 0) {
        return tc_fail(TC_ERR_NOT_IMPLEMENTED, "V7-B scalable packets are not implemented by this library");
    }
    if (n > 45u && memcmp(d, "TPIC", 4u) == 0 && d[6] == 7u && d[45] == 5u) {
        return tc_fail(TC_ERR_UNSUPPORTED_VERSION, "generation 7 (V7-A band decode) retired");
    }
    if (n >= TC_HDR_SIZE && memcmp(d, "TPIC", 4u) == 0 && d[6] == 9u) {
        return tc_fail(TC_ERR_NOT_IMPLEMENTED, "V9 packets are not implemented by this library");
    }
    return 0;
}

static int32_t map_validate(const tc_hdr* h, const tc_shdr* s, uint32_t n)
{
    uint32_t idx = 0;
    for (uint32_t p = 0; p < h->planes; ++p) {
        uint32_t cov = 0;
        const uint32_t rows = h->brows[p];
        while (cov < rows) {
            if (idx >= n) { return tc_fail(TC_ERR_MALFORMED, "plane %u tiling incomplete at block row %u", p, cov); }
            const tc_shdr* x = &s[idx];
            if (x->plane != p) { return tc_fail(TC_ERR_MALFORMED, "slice %u plane %u breaks Y->U->V->[A] order", idx, x->plane); }
            if (x->k1 > 14u || x->k2 > 14u || x->k3 > 14u) { return tc_fail(TC_ERR_MALFORMED, "slice %u k1/k2/k3 > 14", idx); }
            if (h->major == 2u && h->em == 1u && (p < 3u || h->amode == 0u) && (x->k1 > 3u || x->k2 > 3u || x->k3 > 3u)) {
                return tc_fail(TC_ERR_MALFORMED, "slice %u vlc book id > 3", idx);
            }
            if (h->major == 7u && (h->em == 6u || h->em == 7u || h->em == 8u) && (p < 3u || h->amode == 0u) &&
                (x->k1 != 0u || x->k2 != 0u || x->k3 != 0u)) {
                return tc_fail(TC_ERR_MALFORMED, "slice %u rans k1/k2/k3 != 0", idx);
            }
            if (x->y0 != cov) { return tc_fail(TC_ERR_MALFORMED, "slice %u block_y0 %u != expected %u", idx, x->y0, cov); }
            if (x->bh == 0u) { return tc_fail(TC_ERR_MALFORMED, "slice %u block_h == 0", idx); }
            if ((uint32_t)x->y0 + x->bh > rows) { return tc_fail(TC_ERR_MALFORMED, "slice %u band exceeds plane rows %u", idx, rows); }
            const int32_t qp = (int32_t)h->qp + (int32_t)x->qdb - 64;
            if (qp < 0 || qp > (int32_t)TC_QP_MAX) { return tc_fail(TC_ERR_MALFORMED, "slice %u effective qp %d outside 0..95", idx, qp); }
            if (h->amode != 0u && p == 3u && x->k3 != 0u) { return tc_fail(TC_ERR_MALFORMED, "alpha slice %u k3 != 0", idx); }
            cov += x->bh;
            idx++;
        }
    }
    if (idx != n) { return tc_fail(TC_ERR_MALFORMED, "%u trailing slices after full tiling", n - idx); }
    return TC_OK;
}

/* Structural parse from either the whole packet (full != NULL) or from a
 * compact record of its frame header and slice headers (see tcg_device.h,
 * TCG_WALK_REC); both forms apply the same checks in the same order. */
static int32_t parse_impl(const uint8_t* full, const uint8_t* hdr53, const uint8_t* shdrs, size_t n, tc_view* v)
{
    memset(&v->h, 0, sizeof(v->h));
    int32_t rc = hdr_decode(full != NULL ? full : hdr53, n, &v->h);
    if (rc != TC_OK) { return rc; }
    if (v->h.major == 8u || v->h.major == 9u) {
        return tc_fail(TC_ERR_UNSUPPORTED_VERSION, "v8/v9 packet in the V7 scanner");
    }
    if ((uint64_t)v->h.size != (uint64_t)n) { return tc_fail(TC_ERR_MALFORMED, "frame_packet_size %u != actual %zu", v->h.size, n); }
    size_t off = TC_HDR_SIZE;
    for (uint32_t i = 0; i < v->h.slices; ++i) {
        if (off > n || n - off < TC_SH_SIZE) { return tc_fail(TC_ERR_TRUNCATED, "slice %u header out of packet at offset %zu", i, off); }
        const uint8_t* q = full != NULL ? full + off : shdrs + (size_t)i * TC_SH_SIZE;
        tc_shdr* s = &v->s[i];
        s->size = ld32(q); s->plane = q[4]; s->y0 = (uint16_t)ld16(q + 5); s->bh = (uint16_t)ld16(q + 7);
        s->qdb = q[9]; s->k1 = q[10]; s->k2 = q[11]; s->k3 = q[12]; s->crc = ld32(q + 13);
        if (s->k1 > 14u || s->k2 > 14u || s->k3 > 14u) { return tc_fail(TC_ERR_MALFORMED, "slice k1/k2/k3 > 14"); }
        off += TC_SH_SIZE;
        if ((uint64_t)(n - off) < s->size) { return tc_fail(TC_ERR_TRUNCATED, "slice %u payload out of packet", i); }
        v->off[i] = (uint32_t)off;
        off += s->size;
    }
    if (off != n) { return tc_fail(TC_ERR_MALFORMED, "packet has %zu trailing bytes after last slice", n - off); }
    return map_validate(&v->h, v->s, v->h.slices);
}

int32_t tc_parse_structure(const uint8_t* d, size_t n, tc_view* v)
{
    return parse_impl(d, NULL, NULL, n, v);
}

int32_t tc_parse_compact(const uint8_t* rec, size_t n, tc_view* v)
{
    return parse_impl(NULL, rec, rec + 80, n, v);
}

void tc_fill_info(const tc_hdr* h, topos_frame_output* o)
{
    o->visible_width = h->vw; o->visible_height = h->vh;
    o->coded_width = h->cw; o->coded_height = h->ch;
    o->plane_count = h->planes; o->bit_depth = h->bd; o->profile = h->profile;
    o->pixel_format = h->pf; o->alpha_mode = h->amode; o->alpha_bit_depth = h->abd;
    o->color_range = h->range; o->color_primaries = h->prim; o->color_transfer = h->xfer;
    o->color_matrix = h->matrix; o->chroma_siting = h->siting;
    o->sar_num = h->sarn; o->sar_den = h->sard;
    o->slice_count = h->slices;
}
