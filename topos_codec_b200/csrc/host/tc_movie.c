/* tc_movie.c - MOV read path (video track) and its hand-off to the batched
 * GPU decoder.
 *
 * Restates the reference reader for the files its muxer writes
 * (reference: native/src/mov/mov.c): atom walk with bounds checks (:2305-2346),
 * sample-table atoms (:2392-2656), chunk expansion (:2658-2734), sample
 * containment in mdat (:2736-2763), pread reader (:2765-2799), open
 * (:3642-4138), information (:4140-4180), per-sample header checks
 * (:4419-4460), packet reads (:4524-4698), timing and sync (:4700-4753).
 * Audio ('soun') and timecode ('tmcd') tracks are recognised by their
 * handler and skipped without parsing: their own table checks are not made.
 */
#define _POSIX_C_SOURCE 200809L  /* pread */
#include <errno.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>
#include <unistd.h>

#include "../../../include/topos_codec.h"
#include "tc_internal.h"

#define MOV_MDAT_MAX 8
/* movie metadata atom limits (reference topos_codec.h:803-821, mov.c:437-439) */
#define TPCD_VENDOR_MAX 15u
#define TPCD_LABEL_MAX 63u
#define TPCD_PAYLOAD_MAX (12u + TPCD_VENDOR_MAX + TPCD_LABEL_MAX + 4u)
#define TC_TIER_MAX 8u
#define RAW_META_MAX 256u

struct topos_movie {
    topos_io io;
    uint32_t n;                 /* video samples */
    uint32_t timescale;
    uint16_t width, height;
    int faststart;
    uint8_t tpcc_major;
    uint8_t tier;               /* tpcD tier (0 = none) */
    uint8_t budget_set;
    topos_alpha_budget_info budget;
    /* track configuration from tpcC (movie-config fields) */
    uint8_t profile, pf, bd, qm, qp, amode, abd, premul, range, prim, xfer, matrix, siting;
    int8_t dl, dc;
    uint16_t sarn, sard;
    uint64_t* off;
    uint32_t* size;
    uint64_t* pts;
    uint32_t* dur;
    uint8_t* sync;              /* bitmap */
    uint32_t index_bytes;
};

static uint16_t be16(const uint8_t* p) { return (uint16_t)((p[0] << 8) | p[1]); }
static uint32_t be32(const uint8_t* p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }
static uint64_t be64(const uint8_t* p) { return ((uint64_t)be32(p) << 32) | be32(p + 4); }

static int32_t mread(const topos_movie* mv, uint64_t off, void* buf, size_t len)
{
    if (len == 0u) { return TC_OK; }
    if (off > mv->io.length || len > mv->io.length - off) {
        return tc_fail(TC_ERR_TRUNCATED, "io read past the end @%llu+%zu", (unsigned long long)off, len);
    }
    if (mv->io.read(mv->io.ctx, off, buf, len) != TC_OK) { return tc_fail(TC_ERR_IO, "io read failed"); }
    return TC_OK;
}

typedef struct atom {
    uint64_t size, body;
    uint8_t type[4];
    int ext;
} atom;

static int is(const atom* a, const char* t) { return memcmp(a->type, t, 4u) == 0; }
static uint64_t hdr_len(const atom* a) { return a->ext ? 16u : 8u; }

/* atom header at off inside [.., end): 32-bit size, 1 = 64-bit size follows,
 * 0 = to the end of the container */
static int32_t atom_at(const topos_movie* mv, uint64_t off, uint64_t end, atom* a)
{
    if (off > end || end - off < 8u) { return tc_fail(TC_ERR_MALFORMED, "atom header out of bounds"); }
    uint8_t h[8];
    int32_t rc = mread(mv, off, h, 8u);
    if (rc != TC_OK) { return rc; }
    a->size = be32(h);
    memcpy(a->type, h + 4, 4u);
    a->ext = 0;
    a->body = off + 8u;
    if (a->size == 1u) {
        if (end - off < 16u) { return tc_fail(TC_ERR_MALFORMED, "extended size out of bounds"); }
        uint8_t e[8];
        rc = mread(mv, a->body, e, 8u);
        if (rc != TC_OK) { return rc; }
        a->size = be64(e);
        if (a->size < 16u) { return tc_fail(TC_ERR_MALFORMED, "extended size < 16"); }
        a->ext = 1;
        a->body = off + 16u;
    } else if (a->size == 0u) {
        a->size = end - off;
        if (a->size < 8u) { return tc_fail(TC_ERR_MALFORMED, "empty atom"); }
    }
    if (a->size > end - off) { return tc_fail(TC_ERR_MALFORMED, "atom size out of bounds"); }
    return TC_OK;
}

/* full-atom version/flags then an entry count */
static int32_t entries(const topos_movie* mv, uint64_t body, uint64_t end, uint32_t* n)
{
    if (body > end || end - body < 8u) { return tc_fail(TC_ERR_MALFORMED, "full atom too short"); }
    uint8_t b[8];
    const int32_t rc = mread(mv, body, b, 8u);
    if (rc == TC_OK) { *n = be32(b + 4); }
    return rc;
}

typedef struct tables {
    int has_stsd, has_stts, has_stsz, has_stsc, has_stco, has_stss;
    uint32_t stts_n; uint64_t stts_off, stts_end; uint64_t samples;
    uint32_t stsz_uniform, stsz_n; uint64_t stsz_off, stsz_end;
    uint32_t stsc_n; uint64_t stsc_off;
    uint32_t chunks; uint64_t stco_off, stco_end; int co64;
    uint32_t stss_n; uint64_t stss_off, stss_end;
    uint8_t tpcc[28]; int has_tpcc;
    uint8_t tpcb[24]; int has_tpcb;
    int has_tpcd, has_trwm;
    uint16_t w, h;
} tables;

/* the TPIC sample entry and its Topos configuration atoms */
static int32_t read_stsd(topos_movie* mv, uint64_t body, uint64_t end, tables* t)
{
    uint32_t n = 0;
    int32_t rc = entries(mv, body, end, &n);
    if (rc != TC_OK) { return rc; }
    if (n != 1u) { return tc_fail(TC_ERR_MALFORMED, "stsd entry_count=%u != 1", n); }
    atom e;
    rc = atom_at(mv, body + 8u, end, &e);
    if (rc != TC_OK) { return rc; }
    if (!is(&e, "TPIC")) { return tc_fail(TC_ERR_MALFORMED, "not a Topos stream (sample entry is not TPIC)"); }
    if (e.size < hdr_len(&e) + 78u) { return tc_fail(TC_ERR_MALFORMED, "TPIC entry too short"); }
    uint8_t f[70];
    rc = mread(mv, e.body, f, 70u);
    if (rc != TC_OK) { return rc; }
    t->w = be16(f + 24);
    t->h = be16(f + 26);
    const uint64_t eend = e.body + e.size - hdr_len(&e);
    for (uint64_t o = e.body + 78u; o < eend;) {
        atom c;
        rc = atom_at(mv, o, eend, &c);
        if (rc != TC_OK) { return rc; }
        const uint64_t len = c.size - hdr_len(&c);
        if (is(&c, "tpcC")) {
            if (len != 28u) { return tc_fail(TC_ERR_MALFORMED, "tpcC length != 28"); }
            uint8_t p[28];
            rc = mread(mv, c.body, p, 28u);
            if (rc != TC_OK) { return rc; }
            const uint16_t ver = be16(p + 4);
            if (memcmp(p, "TPCC", 4u) != 0 || ver < 1u || ver > 9u) {
                return tc_fail(TC_ERR_MALFORMED, "tpcC magic/version");
            }
            mv->tpcc_major = (uint8_t)ver;
            if (tc_crc32(p, 24u) != be32(p + 24)) { return tc_fail(TC_ERR_CHECKSUM_MISMATCH, "tpcC CRC"); }
            if (t->has_tpcc) { return tc_fail(TC_ERR_MALFORMED, "repeated tpcC"); }
            memcpy(t->tpcc, p, 28u);
            t->has_tpcc = 1;
        } else if (is(&c, "tpcB")) {
            if (len != 24u) { return tc_fail(TC_ERR_MALFORMED, "tpcB length != 24"); }
            uint8_t p[24];
            rc = mread(mv, c.body, p, 24u);
            if (rc != TC_OK) { return rc; }
            if (memcmp(p, "TPCB", 4u) != 0 || be16(p + 4) != 1u) { return tc_fail(TC_ERR_MALFORMED, "tpcB magic/version"); }
            if (tc_crc32(p, 20u) != be32(p + 20)) { return tc_fail(TC_ERR_CHECKSUM_MISMATCH, "tpcB CRC"); }
            if (t->has_tpcb) { return tc_fail(TC_ERR_MALFORMED, "repeated tpcB"); }
            memcpy(t->tpcb, p, 24u);
            t->has_tpcb = 1;
        } else if (is(&c, "tpcD")) {
            if (len < 16u || len > TPCD_PAYLOAD_MAX) { return tc_fail(TC_ERR_MALFORMED, "tpcD length"); }
            uint8_t p[TPCD_PAYLOAD_MAX];
            rc = mread(mv, c.body, p, (size_t)len);
            if (rc != TC_OK) { return rc; }
            if (memcmp(p, "TPCD", 4u) != 0 || be16(p + 4) != 1u) { return tc_fail(TC_ERR_MALFORMED, "tpcD magic/version"); }
            if (p[7] != 0u || p[6] > TC_TIER_MAX) { return tc_fail(TC_ERR_MALFORMED, "tpcD reserved/tier"); }
            const uint32_t vlen = be16(p + 8), llen = be16(p + 10);
            if (12u + (uint64_t)vlen + llen + 4u != len || vlen > TPCD_VENDOR_MAX || llen > TPCD_LABEL_MAX) {
                return tc_fail(TC_ERR_MALFORMED, "tpcD string lengths");
            }
            if (tc_crc32(p, (size_t)(len - 4u)) != be32(p + len - 4u)) {
                return tc_fail(TC_ERR_CHECKSUM_MISMATCH, "tpcD CRC");
            }
            if (t->has_tpcd) { return tc_fail(TC_ERR_MALFORMED, "repeated tpcD"); }
            mv->tier = p[6];
            t->has_tpcd = 1;
        } else if (is(&c, "trwm")) {
            if (len < 8u || len > RAW_META_MAX) { return tc_fail(TC_ERR_MALFORMED, "trwm length"); }
            if (t->has_trwm) { return tc_fail(TC_ERR_MALFORMED, "repeated trwm"); }
            t->has_trwm = 1;
        }
        o += c.size;
    }
    if (!t->has_tpcc) { return tc_fail(TC_ERR_MALFORMED, "missing tpcC"); }
    return TC_OK;
}

static int32_t read_stts(topos_movie* mv, uint64_t body, uint64_t end, tables* t)
{
    uint32_t n = 0;
    int32_t rc = entries(mv, body, end, &n);
    if (rc != TC_OK) { return rc; }
    const uint64_t d = body + 8u, dend = d + (uint64_t)n * 8u;
    if (dend > end) { return tc_fail(TC_ERR_MALFORMED, "stts table out of bounds"); }
    uint64_t total = 0;
    uint8_t blk[4096];
    for (uint64_t o = d; o < dend;) {
        size_t k = (size_t)(dend - o > sizeof(blk) ? sizeof(blk) : dend - o);
        k -= k % 8u;
        rc = mread(mv, o, blk, k);
        if (rc != TC_OK) { return rc; }
        for (size_t i = 0; i < k; i += 8u) {
            if (be32(blk + i + 4) == 0u) { return tc_fail(TC_ERR_MALFORMED, "stts delta 0"); }
            total += be32(blk + i);
        }
        o += k;
    }
    t->stts_n = n;
    t->stts_off = d;
    t->stts_end = dend;
    t->samples = total;
    return TC_OK;
}

static int32_t read_stsz(topos_movie* mv, uint64_t body, uint64_t end, tables* t)
{
    if (body > end || end - body < 12u) { return tc_fail(TC_ERR_MALFORMED, "stsz too short"); }
    uint8_t b[12];
    const int32_t rc = mread(mv, body, b, 12u);
    if (rc != TC_OK) { return rc; }
    t->stsz_uniform = be32(b + 4);
    t->stsz_n = be32(b + 8);
    t->stsz_off = body + 12u;
    t->stsz_end = t->stsz_off + (uint64_t)t->stsz_n * 4u;
    if (t->stsz_uniform == 0u && t->stsz_end > end) { return tc_fail(TC_ERR_MALFORMED, "stsz table out of bounds"); }
    return TC_OK;
}

static int32_t read_table(topos_movie* mv, uint64_t body, uint64_t end, uint32_t esize, uint32_t* n, uint64_t* off,
                          uint64_t* tend, const char* name)
{
    const int32_t rc = entries(mv, body, end, n);
    if (rc != TC_OK) { return rc; }
    *off = body + 8u;
    *tend = *off + (uint64_t)(*n) * esize;
    if (*tend > end) { return tc_fail(TC_ERR_MALFORMED, "%s table out of bounds", name); }
    return TC_OK;
}

/* sample offsets from the chunk table and the samples-per-chunk runs */
static int32_t expand_offsets(topos_movie* mv, const tables* t)
{
    const uint32_t esz = t->co64 ? 8u : 4u;
    uint32_t chunk = 0, si = 0;
    uint64_t coff = t->stco_off;
    uint8_t blk[4096];
    size_t used = 0, pos = 0;
    int32_t rc;
    for (uint32_t e = 0; e < t->stsc_n && si < mv->n; ++e) {
        uint8_t r[12];
        rc = mread(mv, t->stsc_off + (uint64_t)e * 12u, r, 12u);
        if (rc != TC_OK) { return rc; }
        const uint32_t first = be32(r), per = be32(r + 4);
        uint32_t next = 0;
        if (e + 1u < t->stsc_n) {
            uint8_t r2[12];
            rc = mread(mv, t->stsc_off + (uint64_t)(e + 1u) * 12u, r2, 12u);
            if (rc != TC_OK) { return rc; }
            next = be32(r2);
            if (next <= first) { return tc_fail(TC_ERR_MALFORMED, "stsc first_chunk not increasing"); }
        }
        if (first < 1u || per == 0u || first != chunk + 1u) {
            return tc_fail(TC_ERR_MALFORMED, "stsc entry invalid or not contiguous");
        }
        const uint64_t run = e + 1u < t->stsc_n ? (uint64_t)(next - first) : UINT64_MAX;
        for (uint64_t c = 0; c < run && si < mv->n; ++c) {
            if (chunk >= t->chunks) { return tc_fail(TC_ERR_MALFORMED, "stco too few entries"); }
            if (pos >= used) {
                if (coff >= t->stco_end) { return tc_fail(TC_ERR_MALFORMED, "stco data short"); }
                size_t k = (size_t)(t->stco_end - coff > sizeof(blk) ? sizeof(blk) : t->stco_end - coff);
                k -= k % esz;
                if (k == 0u) { return tc_fail(TC_ERR_MALFORMED, "stco tail"); }
                rc = mread(mv, coff, blk, k);
                if (rc != TC_OK) { return rc; }
                used = k;
                pos = 0;
                coff += k;
            }
            uint64_t o = t->co64 ? be64(blk + pos) : be32(blk + pos);
            pos += esz;
            chunk++;
            for (uint32_t k = 0; k < per && si < mv->n; ++k) {
                mv->off[si] = o;
                o += mv->size[si];
                si++;
            }
        }
    }
    if (si != mv->n || chunk != t->chunks) { return tc_fail(TC_ERR_MALFORMED, "stsc/stco do not cover the samples"); }
    return TC_OK;
}

static int32_t read_u32_run(topos_movie* mv, uint64_t off, uint64_t end, uint32_t n, uint32_t* out, const char* name)
{
    uint8_t blk[4096];
    uint32_t i = 0;
    while (i < n) {
        if (off >= end) { return tc_fail(TC_ERR_MALFORMED, "%s data short", name); }
        size_t k = (size_t)(end - off > sizeof(blk) ? sizeof(blk) : end - off);
        k -= k % 4u;
        if (k == 0u) { return tc_fail(TC_ERR_MALFORMED, "%s tail", name); }
        const int32_t rc = mread(mv, off, blk, k);
        if (rc != TC_OK) { return rc; }
        for (size_t p = 0; p < k && i < n; p += 4u) { out[i++] = be32(blk + p); }
        off += k;
    }
    return TC_OK;
}

TC_EXPORT void tc_movie_close(topos_movie* mv)
{
    if (mv == NULL) { return; }
    free(mv->off);
    free(mv->size);
    free(mv->pts);
    free(mv->dur);
    free(mv->sync);
    free(mv);
}

static int32_t open_fail(topos_movie* mv, int32_t rc)
{
    tc_movie_close(mv);
    return rc;
}

/* one video trak: timescale, handler, sample tables */
static int32_t read_video_trak(topos_movie* mv, uint64_t body, uint64_t end, tables* t, int* vide, int* stbl)
{
    int32_t rc;
    for (uint64_t o = body; o < end;) {
        atom a;
        if ((rc = atom_at(mv, o, end, &a)) != TC_OK) { return rc; }
        if (is(&a, "edts")) { return tc_fail(TC_ERR_MALFORMED, "edts/elst not allowed on the video trak"); }
        if (is(&a, "mdia")) {
            const uint64_t mend = o + a.size;
            for (uint64_t d = a.body; d < mend;) {
                atom m;
                if ((rc = atom_at(mv, d, mend, &m)) != TC_OK) { return rc; }
                if (is(&m, "mdhd")) {
                    if (m.size < 32u) { return tc_fail(TC_ERR_MALFORMED, "mdhd too short"); }
                    uint8_t b[8];
                    if ((rc = mread(mv, m.body + 12u, b, 8u)) != TC_OK) { return rc; }
                    mv->timescale = be32(b);
                    if (mv->timescale == 0u) { return tc_fail(TC_ERR_MALFORMED, "timescale 0"); }
                } else if (is(&m, "hdlr")) {
                    if (m.size >= 24u) {
                        uint8_t b[4];
                        if ((rc = mread(mv, m.body + 8u, b, 4u)) != TC_OK) { return rc; }
                        if (memcmp(b, "vide", 4u) == 0) { *vide = 1; }
                    }
                } else if (is(&m, "minf")) {
                    const uint64_t fend = d + m.size;
                    for (uint64_t f = m.body; f < fend;) {
                        atom s;
                        if ((rc = atom_at(mv, f, fend, &s)) != TC_OK) { return rc; }
                        if (is(&s, "stbl")) {
                            *stbl = 1;
                            const uint64_t send = f + s.size;
                            for (uint64_t x = s.body; x < send;) {
                                atom c;
                                if ((rc = atom_at(mv, x, send, &c)) != TC_OK) { return rc; }
                                const uint64_t cend = x + c.size;
                                int* seen = NULL;
                                rc = TC_OK;
                                if (is(&c, "stsd")) {
                                    seen = &t->has_stsd;
                                    if (!*seen) { rc = read_stsd(mv, c.body, cend, t); }
                                } else if (is(&c, "stts")) {
                                    seen = &t->has_stts;
                                    if (!*seen) { rc = read_stts(mv, c.body, cend, t); }
                                } else if (is(&c, "stsz")) {
                                    seen = &t->has_stsz;
                                    if (!*seen) { rc = read_stsz(mv, c.body, cend, t); }
                                } else if (is(&c, "stsc")) {
                                    seen = &t->has_stsc;
                                    uint64_t tend = 0;
                                    if (!*seen) { rc = read_table(mv, c.body, cend, 12u, &t->stsc_n, &t->stsc_off, &tend, "stsc"); }
                                } else if (is(&c, "stco") || is(&c, "co64")) {
                                    seen = &t->has_stco;
                                    if (!*seen) {
                                        t->co64 = is(&c, "co64");
                                        rc = read_table(mv, c.body, cend, t->co64 ? 8u : 4u, &t->chunks, &t->stco_off,
                                                        &t->stco_end, "stco/co64");
                                    }
                                } else if (is(&c, "stss")) {
                                    seen = &t->has_stss;
                                    if (!*seen) {
                                        rc = read_table(mv, c.body, cend, 4u, &t->stss_n, &t->stss_off, &t->stss_end,
                                                        "stss");
                                    }
                                }
                                if (seen != NULL) {
                                    if (*seen) { return tc_fail(TC_ERR_MALFORMED, "repeated sample table atom"); }
                                    *seen = 1;
                                }
                                if (rc != TC_OK) { return rc; }
                                x += c.size;
                            }
                        }
                        f += s.size;
                    }
                }
                d += m.size;
            }
        }
        o += a.size;
    }
    return TC_OK;
}

/* handler type of a trak (mdia > hdlr), zero when it has none */
static int32_t trak_handler(const topos_movie* mv, uint64_t body, uint64_t end, uint8_t out[4])
{
    memset(out, 0, 4u);
    int32_t rc;
    for (uint64_t o = body; o < end;) {
        atom a;
        if ((rc = atom_at(mv, o, end, &a)) != TC_OK) { return rc; }
        if (is(&a, "mdia")) {
            const uint64_t mend = o + a.size;
            for (uint64_t d = a.body; d < mend;) {
                atom m;
                if ((rc = atom_at(mv, d, mend, &m)) != TC_OK) { return rc; }
                if (is(&m, "hdlr") && m.size - hdr_len(&m) >= 12u) { return mread(mv, m.body + 8u, out, 4u); }
                d += m.size;
            }
        }
        o += a.size;
    }
    return TC_OK;
}

TC_EXPORT int32_t tc_movie_open(const topos_io* io, topos_movie** out)
{
    if (io == NULL || out == NULL || io->read == NULL || io->struct_size != (uint32_t)sizeof(topos_io) ||
        io->abi_version != TOPOS_CODEC_ABI_VERSION) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "io NULL, wrong struct_size/abi_version or no read");
    }
    *out = NULL;
    if (io->length < 20u) { return tc_fail(TC_ERR_TRUNCATED, "file too short"); }
    topos_movie* mv = (topos_movie*)calloc(1, sizeof(topos_movie));
    if (mv == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "movie"); }
    mv->io = *io;
    int32_t rc;
    /* top level: ftyp, one moov, up to 8 mdat (a last mdat may run past the end of a truncated file) */
    uint64_t moov_off = UINT64_MAX, moov_end = 0, moov_body = 0, mdat_off = UINT64_MAX;
    uint64_t lo[MOV_MDAT_MAX], hi[MOV_MDAT_MAX];
    int nmdat = 0, ftyp = 0;
    uint64_t off = 0;
    while (off + 8u <= io->length) {
        atom a;
        uint64_t declared_end = 0;
        int truncated = 0;
        rc = atom_at(mv, off, io->length, &a);
        if (rc != TC_OK) {
            uint8_t h8[8];
            if (mread(mv, off, h8, 8u) != TC_OK || memcmp(h8 + 4, "mdat", 4u) != 0) { return open_fail(mv, rc); }
            a.size = io->length - off;
            a.ext = 0;
            a.body = off + 8u;
            memcpy(a.type, "mdat", 4u);
            truncated = 1;
            if (be32(h8) == 1u) {
                uint8_t e8[8];
                if (mread(mv, off + 8u, e8, 8u) == TC_OK) {
                    const uint64_t d = be64(e8);
                    if (d >= 16u && off <= UINT64_MAX - d) { declared_end = off + d; }
                }
            }
            if (declared_end == 0u) { declared_end = io->length; }
        }
        if (is(&a, "ftyp")) {
            ftyp = 1;
        } else if (is(&a, "moov")) {
            if (moov_off != UINT64_MAX) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "repeated moov")); }
            moov_off = off;
            moov_end = off + a.size;
            moov_body = a.body;
        } else if (is(&a, "mdat")) {
            mdat_off = off;
            if (nmdat >= MOV_MDAT_MAX) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "more than 8 mdat")); }
            lo[nmdat] = a.body;
            hi[nmdat] = truncated ? declared_end : off + a.size;
            nmdat++;
        }
        off += a.size;
    }
    if (off != io->length) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "top-level atoms do not close")); }
    if (!ftyp || moov_off == UINT64_MAX) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "missing ftyp or moov")); }
    if (nmdat == 0) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "missing mdat")); }
    mv->faststart = mdat_off != UINT64_MAX && moov_off < mdat_off;

    tables t;
    memset(&t, 0, sizeof(t));
    int have_trak = 0, vide = 0, stbl = 0;
    for (uint64_t o = moov_body; o < moov_end;) {
        atom a;
        if ((rc = atom_at(mv, o, moov_end, &a)) != TC_OK) { return open_fail(mv, rc); }
        if (is(&a, "trak")) {
            uint8_t ht[4];
            if ((rc = trak_handler(mv, a.body, o + a.size, ht)) != TC_OK) { return open_fail(mv, rc); }
            if (memcmp(ht, "soun", 4u) != 0 && memcmp(ht, "tmcd", 4u) != 0) {
                if (have_trak) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "more than one video trak")); }
                have_trak = 1;
                if ((rc = read_video_trak(mv, a.body, o + a.size, &t, &vide, &stbl)) != TC_OK) { return open_fail(mv, rc); }
            }
        }
        o += a.size;
    }
    if (!have_trak || !vide || !stbl) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "moov without trak/vide/stbl")); }
    if (t.samples == 0u) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "empty stts")); }
    if (t.samples > TC_MOVIE_MAX_SAMPLES) { return open_fail(mv, tc_fail(TC_ERR_LIMIT_EXCEEDED, "too many samples")); }
    if ((uint64_t)t.stsz_n != t.samples) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "stsz count != stts samples")); }
    mv->n = (uint32_t)t.samples;
    const size_t n = mv->n;
    mv->off = (uint64_t*)malloc(n * sizeof(uint64_t));
    mv->size = (uint32_t*)malloc(n * sizeof(uint32_t));
    mv->pts = (uint64_t*)malloc(n * sizeof(uint64_t));
    mv->dur = (uint32_t*)malloc(n * sizeof(uint32_t));
    mv->sync = (uint8_t*)calloc(n / 8u + 1u, 1u);
    if (!mv->off || !mv->size || !mv->pts || !mv->dur || !mv->sync) {
        return open_fail(mv, tc_fail(TC_ERR_OUT_OF_MEMORY, "movie index"));
    }
    mv->index_bytes = (uint32_t)(n * (2u * sizeof(uint64_t) + 2u * sizeof(uint32_t)) + n / 8u + 1u);
    {   /* presentation times from the time-to-sample runs */
        uint8_t blk[4096];
        uint64_t p = t.stts_off, acc = 0;
        uint32_t si = 0;
        while (si < mv->n) {
            if (p >= t.stts_end) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "stts short")); }
            size_t k = (size_t)(t.stts_end - p > sizeof(blk) ? sizeof(blk) : t.stts_end - p);
            k -= k % 8u;
            if (k == 0u) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "stts tail")); }
            if ((rc = mread(mv, p, blk, k)) != TC_OK) { return open_fail(mv, rc); }
            for (size_t q = 0; q < k && si < mv->n; q += 8u) {
                const uint32_t cnt = be32(blk + q), d = be32(blk + q + 4);
                for (uint32_t j = 0; j < cnt && si < mv->n; ++j) {
                    mv->pts[si] = acc;
                    mv->dur[si] = d;
                    acc += d;
                    si++;
                }
            }
            p += k;
        }
    }
    if (t.stsz_uniform != 0u) {
        for (uint32_t i = 0; i < mv->n; ++i) { mv->size[i] = t.stsz_uniform; }
    } else {
        if ((rc = read_u32_run(mv, t.stsz_off, t.stsz_end, mv->n, mv->size, "stsz")) != TC_OK) { return open_fail(mv, rc); }
        for (uint32_t i = 0; i < mv->n; ++i) {
            if (mv->size[i] == 0u) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "stsz size 0")); }
        }
    }
    if ((rc = expand_offsets(mv, &t)) != TC_OK) { return open_fail(mv, rc); }
    for (uint32_t i = 0; i < mv->n; ++i) {  /* every sample inside one mdat payload */
        int inside = 0;
        for (int r = 0; r < nmdat && !inside; ++r) {
            inside = mv->off[i] >= lo[r] && mv->off[i] < hi[r] && (uint64_t)mv->size[i] <= hi[r] - mv->off[i];
        }
        if (!inside) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "video sample %u outside mdat", i)); }
    }
    if (t.has_stss) {
        uint32_t* ss = (uint32_t*)malloc((size_t)t.stss_n * 4u + 4u);
        if (ss == NULL) { return open_fail(mv, tc_fail(TC_ERR_OUT_OF_MEMORY, "stss")); }
        rc = read_u32_run(mv, t.stss_off, t.stss_end, t.stss_n, ss, "stss");
        for (uint32_t i = 0; i < t.stss_n && rc == TC_OK; ++i) {
            if (ss[i] < 1u || ss[i] > mv->n) {
                rc = tc_fail(TC_ERR_MALFORMED, "stss out of range");
                break;
            }
            mv->sync[(ss[i] - 1u) / 8u] |= (uint8_t)(1u << ((ss[i] - 1u) % 8u));
        }
        free(ss);
        if (rc != TC_OK) { return open_fail(mv, rc); }
    } else {
        memset(mv->sync, 0xFF, n / 8u + 1u);
    }
    {   /* track configuration (tpcC) checked as a frame configuration of the entry's size */
        const uint8_t* p = t.tpcc;
        mv->profile = p[6]; mv->pf = p[7]; mv->bd = p[8]; mv->qm = p[9]; mv->qp = p[10];
        mv->amode = p[11]; mv->abd = p[12];
        mv->premul = (p[13] & 1u) != 0u;
        mv->range = (p[13] & 2u) != 0u;
        mv->prim = p[14]; mv->xfer = p[15]; mv->matrix = p[16]; mv->siting = p[17];
        mv->sarn = be16(p + 18);
        mv->sard = be16(p + 20);
        topos_frame_config fc;
        memset(&fc, 0, sizeof(fc));
        fc.struct_size = (uint32_t)sizeof(fc);
        fc.abi_version = TOPOS_CODEC_ABI_VERSION;
        fc.visible_width = t.w;
        fc.visible_height = t.h;
        fc.profile = mv->profile;
        fc.pixel_format = mv->pf;
        fc.bit_depth = mv->bd;
        if (mv->bd == 16u) { fc.reserved[0] = 8u; }
        fc.qmatrix_id = mv->qm;
        fc.qp_base = mv->qp;
        fc.slice_rows = 16u;
        fc.alpha_mode = mv->amode;
        fc.alpha_bit_depth = mv->abd;
        fc.alpha_premultiplied = mv->premul;
        fc.color_range = mv->range;
        fc.color_primaries = mv->prim;
        fc.color_transfer = mv->xfer;
        fc.color_matrix = mv->matrix;
        fc.chroma_siting = mv->siting;
        fc.sar_num = mv->sarn;
        fc.sar_den = mv->sard;
        if ((rc = tc_frame_config_validate(&fc)) != TC_OK) { return open_fail(mv, rc); }
        mv->width = t.w;
        mv->height = t.h;
        if (mv->sarn == 0u && mv->sard == 0u) { mv->sarn = mv->sard = 1u; }
    }
    if (t.has_tpcb) {
        if (t.tpcb[6] != mv->amode || t.tpcb[7] != mv->abd) {
            return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "tpcB alpha mode/bit depth differ from tpcC"));
        }
        if (be32(t.tpcb + 16) != mv->n) { return open_fail(mv, tc_fail(TC_ERR_MALFORMED, "tpcB frame_count != samples")); }
        mv->budget.target_ratio_bp = be16(t.tpcb + 8);
        mv->budget.actual_ratio_bp = be16(t.tpcb + 10);
        mv->budget.max_abs_error = be16(t.tpcb + 12);
        mv->budget.flags = be16(t.tpcb + 14);
        mv->budget.frame_count = be32(t.tpcb + 16);
        mv->budget_set = 1u;
    }
    *out = mv;
    return TC_OK;
}

static int32_t fd_read(void* ctx, uint64_t offset, void* buf, size_t len)
{
    const int fd = (int)(intptr_t)ctx;
    uint8_t* p = (uint8_t*)buf;
    size_t got = 0;
    while (got < len) {
        const ssize_t r = pread(fd, p + got, len - got, (off_t)(offset + got));
        if (r < 0 && errno == EINTR) { continue; }
        if (r <= 0) { return TC_ERR_IO; }
        got += (size_t)r;
    }
    return TC_OK;
}

TC_EXPORT int32_t tc_movie_open_fd(int fd, uint64_t length, topos_movie** out)
{
    if (fd < 0 || out == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "fd < 0 or out NULL"); }
    topos_io io;
    memset(&io, 0, sizeof(io));
    io.struct_size = (uint32_t)sizeof(io);
    io.abi_version = TOPOS_CODEC_ABI_VERSION;
    io.ctx = (void*)(intptr_t)fd;
    io.read = fd_read;
    io.length = length;
    return tc_movie_open(&io, out);
}

TC_EXPORT int32_t tc_movie_info(const topos_movie* mv, topos_movie_info* info)
{
    if (mv == NULL || info == NULL || info->struct_size != (uint32_t)sizeof(topos_movie_info) ||
        info->abi_version != TOPOS_CODEC_ABI_VERSION) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "info NULL or wrong struct_size/abi_version");
    }
    memset(info->reserved, 0, sizeof(info->reserved));
    info->visible_width = mv->width;
    info->visible_height = mv->height;
    info->profile = mv->profile;
    info->pixel_format = mv->pf;
    info->bit_depth = mv->bd;
    info->qmatrix_id = mv->qm;
    info->qp_base = mv->qp;
    info->qp_delta_luma = mv->dl;
    info->qp_delta_chroma = mv->dc;
    info->alpha_mode = mv->amode;
    info->alpha_bit_depth = mv->abd;
    info->alpha_premultiplied = mv->premul;
    info->color_range = mv->range;
    info->color_primaries = mv->prim;
    info->color_transfer = mv->xfer;
    info->color_matrix = mv->matrix;
    info->chroma_siting = mv->siting;
    info->sar_num = mv->sarn;
    info->sar_den = mv->sard;
    info->timescale = mv->timescale;
    info->sample_count = mv->n;
    info->faststart = (uint32_t)mv->faststart;
    info->index_bytes = mv->index_bytes;
    info->reserved[0] = mv->tpcc_major;
    info->reserved[1] = mv->tier;
    return TC_OK;
}

TC_EXPORT int32_t tc_movie_alpha_budget(const topos_movie* mv, topos_alpha_budget_info* info)
{
    if (mv == NULL || info == NULL || info->struct_size != (uint32_t)sizeof(topos_alpha_budget_info) ||
        info->abi_version != TOPOS_CODEC_ABI_VERSION) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "info NULL or wrong struct_size/abi_version");
    }
    if (!mv->budget_set) { return tc_fail(TC_ERR_STATE, "movie carries no tpcB alpha budget"); }
    const uint32_t ss = info->struct_size, av = info->abi_version;
    *info = mv->budget;
    info->struct_size = ss;
    info->abi_version = av;
    return TC_OK;
}

/* a sample's header must be a complete packet of the track's configuration */
static int32_t check_sample(const topos_movie* mv, uint32_t i, const uint8_t* p, size_t n)
{
    if (p == NULL || n < TC_HDR_SIZE) { return tc_fail(TC_ERR_TRUNCATED, "sample %u shorter than a frame header", i); }
    int32_t rc = tc_probe_generation(p, n);
    if (rc != TC_OK) { return rc; }
    tc_view* v = (tc_view*)malloc(sizeof(tc_view));
    if (v == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "sample view"); }
    rc = tc_parse_structure(p, n, v);
    if (rc == TC_OK) {
        const tc_hdr* h = &v->h;
        const uint32_t sn = (h->sarn == 0u && h->sard == 0u) ? 1u : h->sarn;
        const uint32_t sd = (h->sarn == 0u && h->sard == 0u) ? 1u : h->sard;
        if ((uint64_t)h->size != (uint64_t)n) {
            rc = tc_fail(TC_ERR_MALFORMED, "sample %u frame_packet_size %u != stsz %zu", i, h->size, n);
        } else if (h->major != mv->tpcc_major || h->vw != mv->width || h->vh != mv->height ||
                   h->profile != mv->profile || h->pf != mv->pf || h->bd != mv->bd || h->qm != mv->qm ||
                   h->amode != mv->amode || h->abd != mv->abd || ((h->flags & 1u) != 0u) != (mv->premul != 0u) ||
                   h->range != mv->range || h->prim != mv->prim || h->xfer != mv->xfer || h->matrix != mv->matrix ||
                   h->siting != mv->siting || sn != mv->sarn || sd != mv->sard) {
            rc = tc_fail(TC_ERR_MALFORMED, "sample %u header differs from the track configuration", i);
        }
    }
    free(v);
    return rc;
}

TC_EXPORT int32_t tc_movie_packet(const topos_movie* mv, uint32_t i, uint8_t* buf, size_t cap, size_t* need)
{
    if (mv == NULL || i >= mv->n) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "sample index out of range"); }
    const size_t sz = mv->size[i];
    if (need != NULL) { *need = sz; }
    const uint64_t off = mv->off[i];
    if (off > mv->io.length || sz > mv->io.length - off) {
        return tc_fail(TC_ERR_MALFORMED, "sample %u range past the end of the file", i);
    }
    if (buf == NULL || cap < sz) { return TC_ERR_BUFFER_TOO_SMALL; }
    const int32_t rc = mread(mv, off, buf, sz);
    return rc != TC_OK ? rc : check_sample(mv, i, buf, sz);
}

/* V7-R2 samples are their own base packets */
TC_EXPORT int32_t tc_movie_packet_base(const topos_movie* mv, uint32_t i, uint8_t* buf, size_t cap, size_t* need)
{
    return tc_movie_packet(mv, i, buf, cap, need);
}

TC_EXPORT int32_t tc_movie_packet_batch(const topos_movie* mv, uint32_t start, uint32_t count, uint8_t* arena,
                                        size_t cap, size_t* offsets_out, size_t* sizes_out, size_t* need_total)
{
    if (mv == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "movie NULL"); }
    if (count == 0u) { return TC_OK; }
    if (start >= mv->n || count > mv->n - start) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "sample range out of range"); }
    uint64_t total = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const uint64_t off = mv->off[start + i], sz = mv->size[start + i];
        if (off > mv->io.length || sz > mv->io.length - off) {
            return tc_fail(TC_ERR_MALFORMED, "sample %u range past the end of the file", start + i);
        }
        if (offsets_out != NULL) { offsets_out[i] = (size_t)total; }
        if (sizes_out != NULL) { sizes_out[i] = (size_t)sz; }
        total += sz;
    }
    if (need_total != NULL) { *need_total = (size_t)total; }
    if (arena == NULL || cap < total) { return TC_ERR_BUFFER_TOO_SMALL; }
    int contiguous = 1;
    for (uint32_t i = 1; i < count && contiguous; ++i) {
        contiguous = mv->off[start + i] == mv->off[start + i - 1u] + mv->size[start + i - 1u];
    }
    int32_t rc = TC_OK;
    if (contiguous) {
        rc = mread(mv, mv->off[start], arena, (size_t)total);  /* one read for the whole range */
    } else {
        size_t p = 0;
        for (uint32_t i = 0; i < count && rc == TC_OK; ++i) {
            rc = mread(mv, mv->off[start + i], arena + p, mv->size[start + i]);
            p += mv->size[start + i];
        }
    }
    size_t p = 0;
    for (uint32_t i = 0; i < count && rc == TC_OK; ++i) {
        rc = check_sample(mv, start + i, arena + p, mv->size[start + i]);
        p += mv->size[start + i];
    }
    return rc;
}

TC_EXPORT int32_t tc_movie_packet_base_batch(const topos_movie* mv, uint32_t start, uint32_t count, uint8_t* arena,
                                             size_t cap, size_t* offsets_out, size_t* sizes_out, uint8_t* base_flags_out,
                                             size_t* need_total)
{
    const int32_t rc = tc_movie_packet_batch(mv, start, count, arena, cap, offsets_out, sizes_out, need_total);
    if (base_flags_out != NULL && (rc == TC_OK || rc == TC_ERR_BUFFER_TOO_SMALL)) { memset(base_flags_out, 0, count); }
    return rc;
}

TC_EXPORT int32_t tc_movie_packet_pts(const topos_movie* mv, uint32_t i, uint64_t* pts_tick, uint32_t* dur_tick)
{
    if (mv == NULL || i >= mv->n || (pts_tick == NULL && dur_tick == NULL)) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "invalid arguments");
    }
    if (pts_tick != NULL) { *pts_tick = mv->pts[i]; }
    if (dur_tick != NULL) { *dur_tick = mv->dur[i]; }
    return TC_OK;
}

TC_EXPORT int32_t tc_movie_packet_sync(const topos_movie* mv, uint32_t i, uint8_t* is_sync)
{
    if (mv == NULL || is_sync == NULL || i >= mv->n) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "invalid arguments"); }
    *is_sync = (uint8_t)((mv->sync[i / 8u] >> (i % 8u)) & 1u);
    return TC_OK;
}

TC_EXPORT int32_t tc_movie_prev_sync(const topos_movie* mv, uint32_t i, uint32_t* sync_index)
{
    if (mv == NULL || sync_index == NULL || i >= mv->n) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "invalid arguments"); }
    for (uint32_t k = i;; --k) {
        if ((mv->sync[k / 8u] >> (k % 8u)) & 1u) {
            *sync_index = k;
            return TC_OK;
        }
        if (k == 0u) { return tc_fail(TC_ERR_STATE, "no sync sample at or before index %u", i); }
    }
}

/* extension: samples straight into one batched decode */
TC_EXPORT int32_t tcg_movie_decode_batch(const topos_movie* mv, uint32_t start, uint32_t count,
                                         uint16_t* const* planes_out, const size_t* strides, topos_frame_output* infos)
{
    if (mv == NULL) { return tc_fail(TC_ERR_INVALID_ARGUMENT, "movie NULL"); }
    if (count == 0u) { return TC_OK; }
    size_t total = 0;
    int32_t rc = tc_movie_packet_batch(mv, start, count, NULL, 0u, NULL, NULL, &total);
    if (rc != TC_ERR_BUFFER_TOO_SMALL && rc != TC_OK) { return rc; }
    uint8_t* arena = (uint8_t*)malloc(total > 0u ? total : 1u);
    size_t* offs = (size_t*)malloc(sizeof(size_t) * count);
    size_t* sizes = (size_t*)malloc(sizeof(size_t) * count);
    topos_batch_packet* pk = (topos_batch_packet*)malloc(sizeof(topos_batch_packet) * count);
    if (arena == NULL || offs == NULL || sizes == NULL || pk == NULL) {
        free(arena); free(offs); free(sizes); free(pk);
        return tc_fail(TC_ERR_OUT_OF_MEMORY, "movie decode arena");
    }
    rc = tc_movie_packet_batch(mv, start, count, arena, total, offs, sizes, &total);
    if (rc == TC_OK) {
        for (uint32_t i = 0; i < count; ++i) {
            pk[i].data = arena + offs[i];
            pk[i].size = sizes[i];
        }
        rc = tc_frame_decode_batch(pk, count, planes_out, strides, infos);
    }
    free(arena); free(offs); free(sizes); free(pk);
    return rc;
}
