/* tc_v8.c - V8 segmented multi-chain rANS packets on the host side (C11):
 * the structure scan, the tile-table checks, the device job of a frame decode
 * and its per-tile status.
 *
 * Layout (reference bitstream/packet.h:36-82): the 53-byte frame header
 * (major 8, entropy 8, slice count = tiles of all planes), an 8-byte extension
 * (segment blocks log2 in 3..5, tile rows log2 in {0, 4..6}, six zero bytes),
 * then per colour plane [segment directory S x 12: stream offset u32 BE,
 * stream length u32 BE, qp_delta_biased, three zero bytes][tile tables
 * T x 350][segment streams][tile CRCs T x 4 BE]. A tile owns the segments
 * whose first block lies in its rows; its CRC covers its table and its
 * member streams, which are contiguous.
 *
 * Packets in device memory are scanned from a sparse host copy: only the
 * header, the directories, the tables and the CRCs are brought over (a few
 * hundred KB for a 3840x2160 frame), at the offsets they have in the packet.
 */
#include <stdlib.h>
#include <string.h>

#include "../tcg_device.h"
#include "tc_internal.h"

#define V8_EXT 8u
#define V8_DIR 12u
#define V8_TABLE 350u

typedef struct v8_tile {
    uint32_t plane, seg_first, seg_count, table_off, stream_off, stream_bytes, crc;
} v8_tile;

typedef struct v8_view {
    tc_hdr h;
    uint32_t sb_log2, sb, tile_rows;
    uint32_t segs[4], tiles[4], dir_off[4], table_off[4], stream_off[4], crc_off[4];
    uint32_t ntiles;
    v8_tile t[TC_MAX_SLICE_COUNT];
} v8_view;

/* bytes [off, off + n) of the packet readable at d + off: a host packet
 * always is; a device packet's sparse copy gets them on demand */
typedef struct v8_src {
    const uint8_t* dev;  /* device packet, or NULL */
    uint8_t* skel;       /* sparse host copy of a device packet */
} v8_src;

static int32_t fetch(v8_src* s, size_t off, size_t n)
{
    if (s->dev == NULL || n == 0u) { return TC_OK; }
    return tcg_read_device(s->skel + off, s->dev + off, n);
}

static uint32_t ld32(const uint8_t* p)
{
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

static int32_t vfail(int32_t code, const char* what, unsigned long long v)
{
    return tc_fail(code, "v8 packet %s = %llu rejected", what, v);
}

/* segments of tile t: [floor(first block / sb), floor(next tile's first block / sb)) */
static void tile_segs(uint32_t t, uint32_t tile_rows, uint32_t cols, uint32_t blocks, uint32_t sb, uint32_t S,
                      uint32_t* sf, uint32_t* sn)
{
    const uint64_t fb = tile_rows == 0u ? 0u : (uint64_t)t * tile_rows * cols;
    const uint64_t fn = tile_rows == 0u ? (uint64_t)blocks : (uint64_t)(t + 1u) * tile_rows * cols;
    uint32_t a = (uint32_t)(fb / sb), b = (uint32_t)(fn / sb);
    if (a > S) { a = S; }
    if (b > S) { b = S; }
    if (b < a) { b = a; }
    *sf = a;
    *sn = b;
}

/* reference: bitstream/packet.c:103-266 (tc_packet_scan_v8_ex, no CRC check:
 * the decode checks the tile CRCs on the device) */
static int32_t v8_scan(v8_src* src, const uint8_t* d, size_t n, v8_view* v)
{
    memset(v, 0, sizeof(*v));
    int32_t rc = tc_hdr_decode(d, n, &v->h);
    if (rc != TC_OK) { return rc; }
    if (v->h.major != 8u && v->h.major != 9u) { return vfail(TC_ERR_UNSUPPORTED_VERSION, "version_major(not v8/v9)", v->h.major); }
    if ((uint64_t)v->h.size != (uint64_t)n) { return tc_fail(TC_ERR_MALFORMED, "frame_packet_size %u != actual %zu", v->h.size, n); }
    if (n < TC_HDR_SIZE + V8_EXT) { return tc_fail(TC_ERR_TRUNCATED, "v8 ext header out of packet"); }
    const uint8_t* ext = d + TC_HDR_SIZE;
    if (ext[0] < 3u || ext[0] > 5u) { return vfail(TC_ERR_MALFORMED, "segment_blocks_log2", ext[0]); }
    if (ext[1] != 0u && (ext[1] < 4u || ext[1] > 6u)) { return vfail(TC_ERR_MALFORMED, "tile_rows_log2", ext[1]); }
    for (uint32_t i = 2; i < V8_EXT; ++i) {
        if (ext[i] != 0u) { return vfail(TC_ERR_MALFORMED, "ext reserved(!=0)", ext[i]); }
    }
    v->sb_log2 = ext[0];
    v->sb = 1u << ext[0];
    v->tile_rows = ext[1] == 0u ? 0u : 1u << ext[1];
    size_t off = TC_HDR_SIZE + V8_EXT;
    uint32_t nt = 0;
    for (uint32_t p = 0; p < v->h.planes; ++p) {
        const uint32_t rows = v->h.brows[p], cols = v->h.bcols[p], blocks = rows * cols;
        const uint32_t S = (blocks + v->sb - 1u) / v->sb;
        const uint32_t T = (v->tile_rows == 0u || rows == 0u) ? 1u : (rows + v->tile_rows - 1u) / v->tile_rows;
        v->segs[p] = S;
        v->tiles[p] = T;
        v->dir_off[p] = (uint32_t)off;
        if (off > n || (size_t)S * V8_DIR > n - off) { return tc_fail(TC_ERR_TRUNCATED, "v8 plane %u dir out of packet", p); }
        if ((rc = fetch(src, off, (size_t)S * V8_DIR)) != TC_OK) { return rc; }
        off += (size_t)S * V8_DIR;
        v->table_off[p] = (uint32_t)off;
        if (off > n || (size_t)T * V8_TABLE > n - off) { return tc_fail(TC_ERR_TRUNCATED, "v8 plane %u tables out of packet", p); }
        if ((rc = fetch(src, off, (size_t)T * V8_TABLE)) != TC_OK) { return rc; }
        off += (size_t)T * V8_TABLE;
        v->stream_off[p] = (uint32_t)off;
        const uint8_t* dir = d + v->dir_off[p];
        uint64_t sl = 0;
        for (uint32_t k = 0; k < S; ++k) {
            const uint32_t so = ld32(dir + (size_t)k * V8_DIR), ln = ld32(dir + (size_t)k * V8_DIR + 4u);
            if (ln < 4u) { return vfail(TC_ERR_MALFORMED, "segment stream_len(<state)", ln); }
            if (k == 0u) {
                if (so != 0u) { return vfail(TC_ERR_MALFORMED, "seg0 stream_off", so); }
            } else if (so != ld32(dir + (size_t)(k - 1u) * V8_DIR) + ld32(dir + (size_t)(k - 1u) * V8_DIR + 4u)) {
                return vfail(TC_ERR_MALFORMED, "segment dir gap/off", so);
            }
            sl += ln;
            if (sl > TC_MAX_PACKET) { return vfail(TC_ERR_LIMIT_EXCEEDED, "plane stream bytes", sl); }
        }
        if (off > n || sl > n - off) { return tc_fail(TC_ERR_TRUNCATED, "v8 plane %u stream out of packet", p); }
        off += (size_t)sl;
        v->crc_off[p] = (uint32_t)off;
        if (off > n || (size_t)T * 4u > n - off) { return tc_fail(TC_ERR_TRUNCATED, "v8 plane %u crc out of packet", p); }
        if ((rc = fetch(src, off, (size_t)T * 4u)) != TC_OK) { return rc; }
        for (uint32_t t = 0; t < T; ++t) {
            if (nt + t >= TC_MAX_SLICE_COUNT) { return vfail(TC_ERR_MALFORMED, "slice_count(!= tile total)", nt + t); }
            v8_tile* ti = &v->t[nt + t];
            uint32_t sf, sn;
            tile_segs(t, v->tile_rows, cols, blocks, v->sb, S, &sf, &sn);
            ti->plane = p;
            ti->seg_first = sf;
            ti->seg_count = sn - sf;
            ti->table_off = v->table_off[p] + t * V8_TABLE;
            ti->crc = ld32(d + off + (size_t)t * 4u);
            ti->stream_off = v->stream_off[p] + (sn > sf ? ld32(dir + (size_t)sf * V8_DIR) : 0u);
            ti->stream_bytes = 0u;
            for (uint32_t k = sf; k < sn; ++k) { ti->stream_bytes += ld32(dir + (size_t)k * V8_DIR + 4u); }
        }
        nt += T;
        off += (size_t)T * 4u;
    }
    if (off != n) { return tc_fail(TC_ERR_MALFORMED, "v8 packet has %zu trailing bytes", n - off); }
    if (nt != v->h.slices) {
        return vfail(TC_ERR_MALFORMED, "slice_count(!= tile total)", ((unsigned long long)v->h.slices << 16) | nt);
    }
    v->ntiles = nt;
    return TC_OK;
}

/* tile tables of one plane (reference codec.c:4349-4380): flags, and every
 * row the model uses must normalise, which fails only for an all-zero row */
static int32_t check_tables(const uint8_t* d, const v8_view* v, uint32_t p, uint32_t t0)
{
    for (uint32_t t = t0; t < t0 + v->tiles[p]; ++t) {
        const uint8_t* tb = d + v->t[t].table_off;
        const uint32_t fl = tb[0], lm = fl & 3u, dm = (fl >> 2) & 1u;
        if ((fl & 0xF8u) != 0u || lm > 2u) { return tc_fail(TC_ERR_MALFORMED, "v8 tile flags %u", fl); }
        const uint32_t nd = dm ? 5u : 1u, nl = lm == 1u ? 4u : lm == 2u ? 5u : 1u;
        for (uint32_t c = 0; c < nd + 1u + nl; ++c) {
            const uint32_t off = c < nd ? 1u + c * 29u : c == nd ? 146u : 210u + (c - nd - 1u) * 28u;
            const uint32_t len = c < nd ? 29u : c == nd ? 64u : 28u;
            uint32_t sum = 0;
            for (uint32_t k = 0; k < len; ++k) { sum += tb[off + k]; }
            if (sum == 0u) {
                return c < nd ? tc_fail(TC_ERR_MALFORMED, "v8 tile dc row %u", c)
                              : c == nd ? tc_fail(TC_ERR_MALFORMED, "v8 tile run row")
                                        : tc_fail(TC_ERR_MALFORMED, "v8 tile lvl row %u", c - nd - 1u);
            }
        }
    }
    return TC_OK;
}

/* One frame prepared for the device: its view, the job and the job's arrays. */
typedef struct v8_prep {
    v8_src src;
    v8_view* v;
    tcg_v8_seg* seg;
    tcg_v8_tile* tile;
    uint8_t* fail;
    uint32_t* q;
    tcg_v8_job job;
} v8_prep;

static void v8_release(v8_prep* P)
{
    free(P->v);
    free(P->src.skel);
    free(P->seg);
    free(P->tile);
    free(P->fail);
    free(P->q);
    memset(P, 0, sizeof(*P));
}

/* Scan, checks in the reference's order and the device job of one frame
 * (reference codec.c:4772-4870). planes_out NULL: the query only (structure
 * and frame information), *query set. */
static int32_t v8_prepare(const uint8_t* data, size_t size, uint16_t* const planes_out[4], const size_t* strides,
                          topos_frame_output* o, v8_prep* P, int* query)
{
    memset(P, 0, sizeof(*P));
    *query = 0;
    const uint8_t* d = data;
    if (tcg_is_device_ptr(data)) {
        P->src.dev = data;
        P->src.skel = (uint8_t*)malloc(size > 0u ? size : 1u);
        if (P->src.skel == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "v8 packet structure copy"); }
        const int32_t rc = fetch(&P->src, 0u, size < TC_HDR_SIZE + V8_EXT ? size : TC_HDR_SIZE + V8_EXT);
        if (rc != TC_OK) { return rc; }
        d = P->src.skel;
    }
    P->v = (v8_view*)malloc(sizeof(v8_view));
    if (P->v == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "v8 view"); }
    v8_view* v = P->v;
    int32_t rc = v8_scan(&P->src, d, size, v);
    if (rc != TC_OK) { return rc; }
    if (planes_out == NULL) {
        tc_fill_info(&v->h, o);
        *query = 1;
        return TC_OK;
    }
    if (v->h.major == 9u) { return tc_fail(TC_ERR_NOT_IMPLEMENTED, "V9 packets are not implemented by this library"); }
    if (v->h.pf == 3u) { return tc_fail(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "v8 does not carry CFA (TRAW uses rans2)"); }
    tc_fill_info(&v->h, o);
    const tc_hdr* h = &v->h;
    for (uint32_t p = 0; p < h->planes; ++p) {
        if (planes_out[p] == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "v8 planes_out[%u] == NULL", p); }
    }
    uint16_t qm[2][64];
    uint32_t t0 = 0;
    for (uint32_t p = 0; p < h->planes; ++p) {
        if ((rc = check_tables(d, v, p, t0)) != TC_OK) { return rc; }
        t0 += v->tiles[p];
        if (!tc_qmatrix(h->qm, 0, qm[0]) || !tc_qmatrix(h->qm, 1, qm[1])) {
            return tc_fail(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id %u", h->qm);
        }
    }
    for (uint32_t p = 0; p < h->planes; ++p) {
        const size_t s = strides != NULL ? strides[p] : 0u;
        if (s != 0u && s < (size_t)h->pvw[p]) {
            return tc_fail(TC_ERR_INVALID_ARGUMENT, "plane %u stride %zu < visible width %u", p, s, h->pvw[p]);
        }
    }
    uint32_t nseg = 0;
    for (uint32_t p = 0; p < h->planes; ++p) { nseg += v->segs[p]; }
    P->seg = (tcg_v8_seg*)calloc(nseg ? nseg : 1u, sizeof(tcg_v8_seg));
    P->tile = (tcg_v8_tile*)calloc(v->ntiles ? v->ntiles : 1u, sizeof(tcg_v8_tile));
    P->fail = (uint8_t*)calloc(nseg + v->ntiles + 1u, 1);
    P->q = (uint32_t*)malloc(2u * 96u * 64u * sizeof(uint32_t));
    if (P->seg == NULL || P->tile == NULL || P->fail == NULL || P->q == NULL) {
        return tc_fail(TC_ERR_OUT_OF_MEMORY, "v8 decode job");
    }
    tcg_v8_seg* seg = P->seg;
    tcg_v8_tile* tile = P->tile;
    /* quantiser steps per (matrix, effective qp) that a segment uses */
    int32_t qslot[2][96];
    memset(qslot, 0xFF, sizeof(qslot));
    uint32_t nq = 0, k = 0, tg = 0;
    const int32_t ceil = h->qp >= TC_QP_V15_MIN ? (int32_t)TC_QP_MAX : 63;
    const uint32_t refined = (h->flags & 0x8u) != 0u;
    for (uint32_t p = 0; p < h->planes; ++p) {
        const uint32_t blocks = h->brows[p] * h->bcols[p];
        const uint8_t* dir = d + v->dir_off[p];
        const int chroma = p == 1u || p == 2u;
        for (uint32_t s = 0; s < v->segs[p]; ++s, ++k) {
            int32_t qe = (int32_t)h->qp + (int32_t)dir[(size_t)s * V8_DIR + 8u] - 64;
            qe = qe < 0 ? 0 : (qe > ceil ? ceil : qe);
            if (qslot[chroma][qe] < 0) {
                qslot[chroma][qe] = (int32_t)nq;
                tc_quant_steps(qm[chroma], (uint32_t)qe, refined, P->q + (size_t)nq * 64u);
                nq++;
            }
            seg[k].plane = p;
            seg[k].blk0 = s * v->sb;
            seg[k].nblk = blocks - s * v->sb < v->sb ? blocks - s * v->sb : v->sb;
            seg[k].tile = UINT32_MAX;
            seg[k].off = v->stream_off[p] + ld32(dir + (size_t)s * V8_DIR);
            seg[k].len = ld32(dir + (size_t)s * V8_DIR + 4u);
            seg[k].qidx = (uint32_t)qslot[chroma][qe];
        }
        for (uint32_t t = 0; t < v->tiles[p]; ++t, ++tg) {
            const v8_tile* ti = &v->t[tg];
            tile[tg].plane = p;
            tile[tg].seg0 = k - v->segs[p] + ti->seg_first;
            tile[tg].nseg = ti->seg_count;
            tile[tg].table_off = ti->table_off;
            tile[tg].stream_off = ti->stream_off;
            tile[tg].stream_bytes = ti->stream_bytes;
            tile[tg].crc = ti->crc;
            for (uint32_t x = 0; x < ti->seg_count; ++x) { seg[tile[tg].seg0 + x].tile = tg; }
        }
    }
    tcg_v8_job* J = &P->job;
    J->packet = data;
    J->size = size;
    J->bit_depth = h->bd;
    J->sb_log2 = v->sb_log2;
    for (uint32_t p = 0; p < 3u; ++p) {
        J->vis_w[p] = h->pvw[p]; J->vis_h[p] = h->pvh[p];
        J->cols[p] = h->bcols[p]; J->rows[p] = h->brows[p];
        J->dst[p] = planes_out[p];
        J->dst_stride[p] = strides != NULL ? strides[p] : 0u;
    }
    J->nseg = nseg;
    J->ntile = v->ntiles;
    J->nq = nq;
    J->seg = seg;
    J->tile = tile;
    J->q = P->q;
    J->seg_fail = P->fail;
    J->tile_ok = P->fail + nseg;
    return TC_OK;
}

/* per-tile status: concealed when its CRC failed or a member segment failed */
static void v8_status(const v8_prep* P, topos_frame_output* o)
{
    uint32_t concealed = 0;
    for (uint32_t t = 0; t < P->job.ntile; ++t) {
        uint32_t bad = P->job.tile_ok[t] == 0u;
        for (uint32_t s = 0; s < P->tile[t].nseg && !bad; ++s) { bad = P->job.seg_fail[P->tile[t].seg0 + s]; }
        o->slice_status[t] = bad ? TC_FRAME_SLICE_CONCEALED : TC_FRAME_SLICE_OK;
        concealed += bad;
    }
    o->concealed_slices = (uint16_t)concealed;
}

/* reference: codec.c:9039-9049 (tc_frame_decode's V8 branch), 4772-4975
 * (v8_frame_decode). Concealed tiles are reported per tile and counted, and
 * the call still returns TC_OK, as the reference's does; V8 has no
 * deblocking. A segment no tile owns (possible only in a hand-made packet)
 * reconstructs at the mid level here; the reference leaves those samples
 * unwritten. */
int32_t tc_v8_frame_decode(const uint8_t* data, size_t size, uint16_t* const planes_out[4], const size_t strides[4],
                           topos_frame_output* o)
{
    v8_prep P;
    int query = 0;
    int32_t rc = v8_prepare(data, size, planes_out, strides, o, &P, &query);
    if (rc == TC_OK && !query) {
        rc = tcg_decode_v8(&P.job, 1u);
        if (rc == TC_OK) { v8_status(&P, o); }
    }
    v8_release(&P);
    return rc;
}

/* Extension (no reference counterpart; the reference's batch decode takes V7
 * packets only): count V8 packets decoded in one launch sequence. Every
 * packet is scanned and checked first, and any failure fails the call
 * (like tc_frame_decode_batch); planes_out NULL = query only. Returns TC_OK
 * or the first failing packet's status; concealment is reported per tile. */
TC_EXPORT int32_t tcg_frame_decode_v8_batch(const topos_batch_packet* packets, uint32_t count,
                                            uint16_t* const* planes_out, const size_t* strides,
                                            topos_frame_output* infos)
{
    if (count == 0u) { return TC_OK; }
    if (count > TC_BATCH_MAX_FRAMES) { return tc_fail(TC_ERR_LIMIT_EXCEEDED, "batch count %u", count); }
    if (packets == NULL || infos == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "batch arguments NULL"); }
    v8_prep* P = (v8_prep*)calloc(count, sizeof(v8_prep));
    tcg_v8_job* jobs = (tcg_v8_job*)calloc(count, sizeof(tcg_v8_job));
    if (P == NULL || jobs == NULL) {
        free(P);
        free(jobs);
        return tc_fail(TC_ERR_OUT_OF_MEMORY, "v8 batch staging");
    }
    int32_t rc = TC_OK;
    uint32_t prepared = 0;
    for (uint32_t i = 0; i < count && rc == TC_OK; ++i) {
        topos_frame_output* o = &infos[i];
        memset(o, 0, sizeof(*o));
        o->struct_size = (uint32_t)sizeof(topos_frame_output);
        o->abi_version = TOPOS_CODEC_ABI_VERSION;
        int query = 0;
        if (packets[i].data == NULL) {
            rc = tc_fail(TC_ERR_INVALID_ARGUMENT, "packets[%u].data == NULL", i);
        } else if (tc_packet_major(packets[i].data, packets[i].size) != 8) {
            rc = tc_fail(TC_ERR_UNSUPPORTED_VERSION, "packets[%u] is not a V8 packet", i);
        } else {
            rc = v8_prepare(packets[i].data, packets[i].size,
                            planes_out != NULL ? planes_out + (size_t)i * TC_FRAME_MAX_PLANES : NULL,
                            strides != NULL ? strides + (size_t)i * TC_FRAME_MAX_PLANES : NULL, o, &P[i], &query);
        }
        prepared = i + 1u;
        jobs[i] = P[i].job;
    }
    if (rc == TC_OK && planes_out != NULL) {
        rc = tcg_decode_v8(jobs, count);
        for (uint32_t i = 0; i < count && rc == TC_OK; ++i) { v8_status(&P[i], &infos[i]); }
    }
    for (uint32_t i = 0; i < prepared; ++i) { v8_release(&P[i]); }
    free(P);
    free(jobs);
    return rc;
}
