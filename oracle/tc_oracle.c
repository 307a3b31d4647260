/* tc_oracle.c - CPU oracle for the Topos Codec V7-R2 intra frame path.
 *
 * TEST INFRASTRUCTURE ONLY (see tc_oracle.h). A plain, scalar C restatement of
 * the reference algorithm for the frame path, written for clarity rather than
 * speed. Each function cites the reference file:line it follows (paths are
 * relative to the reference project root).
 *
 * Pinning: tests link the reference's own golden conformance driver
 * (native/tests/conformance/golden_codec.c) against this library and check
 * golden_codec_v7r2_intra.bin byte-for-byte, and run seeded differential cases
 * against the reference library built from its sources (oracle/_ref).
 */
#include "tc_oracle.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

/* ============================ limits and constants ============================ */

#define HDR_SIZE 53u            /* frame header bytes   (frame_header.h:15) */
#define SH_SIZE 17u             /* slice header bytes   (slice_map.h:10) */
#define MAX_DIM 16384u          /* frame_header.h:17 */
#define MAX_SLICES 512u         /* frame_header.h:18 */
#define MAX_PACKET 268435456u   /* frame_header.h:19 */
#define QP_MAX 95u              /* quant.h:21 */
#define QP_V15_MIN 64u          /* quant.h:23 */
#define TRAW_LOG0 20u           /* frame_header.h:26 */
#define BATCH_MAX 65536u        /* codec.h:166 */

#define RANS_L (1u << 23)       /* rans.h:27 */
#define RANS_SCALE 4096u        /* rans.h:29 */
#define DC_SYMS 29u             /* rans.h:148 */
#define RUN_SYMS 64u
#define LVL_SYMS 28u
#define POS_CTX 4u              /* rans.h:254-256 */
#define PREV_CTX 5u
#define DCP_CTX 5u

#define M_MAX_DC 0x08000000u          /* rice.h:25 */
#define M_MAX_LVL 0x04000000u         /* rice.h:26 */
#define M_MAX_ALPHA 0x00020000u       /* rice.h:28 */
#define M_MAX_DC_BD16 0x0FFFFFFFu     /* rice.h:51 */
#define M_MAX_LVL_BD16 0x07FFFFFFu    /* rice.h:52 */
#define DC_DOMAIN (1 << 25)           /* rice.h:38 */
#define DC_DOMAIN_BD16 (1 << 27)      /* rice.h:53 */
#define F_MAX (1 << 25)               /* transform.h:8 */
#define F_MAX_WIDE (1 << 30)          /* transform.h:11 */

/* ============================ thread-local error ============================ */
/* reference: native/src/common/error.c:9-31 ("[status] detail") */

static _Thread_local char g_err[256];

static int32_t fail(int32_t st, const char* fmt, ...)
{
    int n = snprintf(g_err, sizeof(g_err), "[%d] ", (int)st);
    if (n < 0) { g_err[0] = 0; return st; }
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err + n, sizeof(g_err) - (size_t)n, fmt, ap);
    va_end(ap);
    return st;
}

EXPORT const char* tc_last_error(void) { return g_err; }

/* ============================ frozen tables ============================ */

/* zigzag scan -> natural index (scan.h:12-21) */
static const uint8_t ZZ[64] = {
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

/* transform basis M[u][x], row energies E[u], inverse weights W[u][v]
 * (transform_tables.h:10-36) */
static const int32_t TM[64] = {
    13, 13, 13, 13, 13, 13, 13, 13, 13, 11, 7, 1, -1, -7, -11, -13,
    12, 5, -5, -12, -12, -5, 5, 12, 11, -4, -13, -8, 8, 13, 4, -11,
    9, -9, -9, 9, 9, -9, -9, 9, 8, -13, 4, 11, -11, -4, 13, -8,
    5, -12, 12, -5, -5, 12, -12, 5, 1, -7, 11, -13, 13, -11, 7, -1};
static const int64_t TE[8] = {1352, 680, 676, 740, 648, 740, 676, 680};
static const int64_t TW[64] = {
    2350, 4672, 4699, 4293, 4902, 4293, 4699, 4672,
    4672, 9288, 9343, 8535, 9747, 8535, 9343, 9288,
    4699, 9343, 9399, 8586, 9805, 8586, 9399, 9343,
    4293, 8535, 8586, 7843, 8957, 7843, 8586, 8535,
    4902, 9747, 9805, 8957, 10228, 8957, 9805, 9747,
    4293, 8535, 8586, 7843, 8957, 7843, 8586, 8535,
    4699, 9343, 9399, 8586, 9805, 8586, 9399, 9343,
    4672, 9288, 9343, 8535, 9747, 8535, 9343, 9288};

/* qp -> scale, classic and refined (quant.c:18-52) */
static const uint32_t QPS[96] = {
    1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5, 6, 7,
    8, 10, 11, 13, 16, 19, 23, 27, 32, 38, 45, 54, 64, 76, 91, 108,
    128, 152, 181, 215, 256, 304, 362, 431, 512, 609, 724, 861, 1024, 1218, 1448, 1722,
    2048, 2435, 2896, 3444, 4096, 4871, 5793, 6889, 8192, 9742, 11585, 13777, 16384, 19484, 23170, 27555,
    32768, 38968, 46341, 55109, 65536, 77936, 92682, 110218,
    131072, 155872, 185364, 220436, 262144, 311744, 370728, 440872,
    524288, 623487, 741455, 881744, 1048576, 1246974, 1482910, 1763488,
    2097152, 2493948, 2965821, 3526975, 4194304, 4987896, 5931642, 7053950};
static const uint32_t QPS_REFINED_HI[32] = {
    32768, 36781, 41285, 46341, 52016, 58386, 65536, 73562,
    82570, 92682, 104032, 116772, 131072, 147123, 165140, 185364,
    208064, 233544, 262144, 294247, 330281, 370728, 416128, 467088,
    524288, 588493, 660561, 741455, 832255, 934175, 1048576, 1176987};

static uint32_t qp_scale(uint32_t refined, uint32_t qp)
{
    if (qp > QP_MAX) { return 0u; }
    if (refined && qp >= 64u) { return QPS_REFINED_HI[qp - 64u]; }
    return QPS[qp];
}

/* quantisation matrices, natural order, luma then chroma (quant.c:54-186).
 * ids 1..3 are geometric tables; id 4 the edge-balanced table. */
static const uint16_t QM_STD_L[64] = {
    16, 20, 25, 31, 39, 49, 61, 76, 20, 25, 31, 39, 49, 61, 76, 95,
    25, 31, 39, 49, 61, 76, 95, 119, 31, 39, 49, 61, 76, 95, 119, 149,
    39, 49, 61, 76, 95, 119, 149, 186, 49, 61, 76, 95, 119, 149, 186, 233,
    61, 76, 95, 119, 149, 186, 233, 291, 76, 95, 119, 149, 186, 233, 291, 364};
static const uint16_t QM_STD_C[64] = {
    16, 19, 22, 26, 31, 37, 43, 51, 19, 22, 26, 31, 37, 43, 51, 60,
    22, 26, 31, 37, 43, 51, 60, 71, 26, 31, 37, 43, 51, 60, 71, 84,
    31, 37, 43, 51, 60, 71, 84, 99, 37, 43, 51, 60, 71, 84, 99, 117,
    43, 51, 60, 71, 84, 99, 117, 138, 51, 60, 71, 84, 99, 117, 138, 162};
static const uint16_t QM_444C_L[64] = {
    16, 36, 45, 56, 70, 88, 110, 137, 36, 45, 56, 70, 88, 110, 137, 171,
    45, 56, 70, 88, 110, 137, 171, 214, 56, 70, 88, 110, 137, 171, 214, 268,
    70, 88, 110, 137, 171, 214, 268, 335, 88, 110, 137, 171, 214, 268, 335, 419,
    110, 137, 171, 214, 268, 335, 419, 524, 137, 171, 214, 268, 335, 419, 524, 655};
static const uint16_t QM_444C_C[64] = {
    16, 28, 33, 39, 46, 56, 64, 76, 28, 33, 39, 46, 56, 64, 76, 90,
    33, 39, 46, 56, 64, 76, 90, 106, 39, 46, 56, 64, 76, 90, 106, 126,
    46, 56, 64, 76, 90, 106, 126, 148, 56, 64, 76, 90, 106, 126, 148, 176,
    64, 76, 90, 106, 126, 148, 176, 207, 76, 90, 106, 126, 148, 176, 207, 243};
static const uint16_t QM_422L_L[64] = {
    16, 22, 27, 33, 42, 53, 66, 82, 22, 27, 33, 42, 53, 66, 82, 103,
    27, 33, 42, 53, 66, 82, 103, 129, 33, 42, 53, 66, 82, 103, 129, 161,
    42, 53, 66, 82, 103, 129, 161, 201, 53, 66, 82, 103, 129, 161, 201, 252,
    66, 82, 103, 129, 161, 201, 252, 314, 82, 103, 129, 161, 201, 252, 314, 393};
static const uint16_t QM_422L_C[64] = {
    16, 20, 23, 27, 33, 39, 45, 54, 20, 23, 27, 33, 39, 45, 54, 63,
    23, 27, 33, 39, 45, 54, 63, 75, 27, 33, 39, 45, 54, 63, 75, 88,
    33, 39, 45, 54, 63, 75, 88, 104, 39, 45, 54, 63, 75, 88, 104, 123,
    45, 54, 63, 75, 88, 104, 123, 145, 54, 63, 75, 88, 104, 123, 145, 170};
static const uint16_t QM_EB_L[64] = {
    20, 19, 18, 17, 16, 15, 14, 13, 19, 18, 17, 16, 15, 14, 13, 12,
    18, 17, 16, 15, 14, 13, 12, 11, 17, 16, 15, 14, 13, 12, 11, 11,
    16, 15, 14, 13, 12, 11, 11, 10, 15, 14, 13, 12, 11, 11, 10, 9,
    14, 13, 12, 11, 11, 10, 9, 9, 13, 12, 11, 11, 10, 9, 9, 8};
static const uint16_t QM_EB_C[64] = {
    18, 17, 16, 16, 15, 14, 13, 13, 17, 16, 16, 15, 14, 13, 13, 12,
    16, 16, 15, 14, 13, 13, 12, 11, 16, 15, 14, 13, 13, 12, 11, 11,
    15, 14, 13, 13, 12, 11, 11, 10, 14, 13, 13, 12, 11, 11, 10, 10,
    13, 13, 12, 11, 11, 10, 10, 9, 13, 12, 11, 11, 10, 10, 9, 9};

/* qmatrix_id -> (luma, chroma) tables; id 0 is flat 16. Returns 0 if unknown. */
static int qm_lookup(uint8_t id, int chroma, uint16_t out[64])
{
    const uint16_t* t = NULL;
    switch (id) {
    case 0: for (int i = 0; i < 64; ++i) { out[i] = 16u; } return 1;
    case 1: t = chroma ? QM_STD_C : QM_STD_L; break;
    case 2: t = chroma ? QM_444C_C : QM_444C_L; break;
    case 3: t = chroma ? QM_422L_C : QM_422L_L; break;
    case 4: t = chroma ? QM_EB_C : QM_EB_L; break;
    default: return 0;
    }
    memcpy(out, t, 64u * sizeof(uint16_t));
    return 1;
}

/* ============================ small helpers ============================ */

static void be16(uint8_t* p, uint32_t v) { p[0] = (uint8_t)(v >> 8); p[1] = (uint8_t)v; }
static void be32(uint8_t* p, uint32_t v)
{
    p[0] = (uint8_t)(v >> 24); p[1] = (uint8_t)(v >> 16);
    p[2] = (uint8_t)(v >> 8); p[3] = (uint8_t)v;
}
static uint32_t ld16(const uint8_t* p) { return ((uint32_t)p[0] << 8) | p[1]; }
static uint32_t ld32(const uint8_t* p)
{
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

static uint32_t bitlen(uint32_t m) { return m == 0u ? 0u : 32u - (uint32_t)__builtin_clz(m); }

/* signed <-> unsigned map (rice.c:3-17) */
static uint32_t map_s(int32_t v)
{
    int64_t s = v;
    return s >= 0 ? (uint32_t)((uint64_t)s << 1) : (uint32_t)(((uint64_t)(-s) << 1) - 1u);
}
static int32_t unmap_s(uint32_t m)
{
    uint64_t u = m;
    return (u & 1u) == 0u ? (int32_t)(u / 2u) : -(int32_t)((u + 1u) / 2u);
}

/* DC predictor (block_coding.c:7-18) */
static int32_t dc_pred(int has_l, int32_t l, int has_t, int32_t t)
{
    if (has_l && has_t) {
        int64_t s = (int64_t)l + t;
        return s >= 0 ? (int32_t)((s + 1) >> 1) : -(int32_t)((-s) >> 1);
    }
    if (has_l) { return l; }
    if (has_t) { return t; }
    return 0;
}

/* MED predictor (codec.h:18-23) */
static int32_t med(int32_t a, int32_t b, int32_t c)
{
    if (c >= a && c >= b) { return a < b ? a : b; }
    if (c <= a && c <= b) { return a < b ? b : a; }
    return a + b - c;
}

static int32_t rshift32_round(int64_t v)
{
    if (v >= 0) { return (int32_t)((v + ((int64_t)1 << 31)) >> 32); }
    return -(int32_t)((-v + ((int64_t)1 << 31)) >> 32);
}

/* ============================ CRC-32 ============================ */

static uint32_t g_crc_tab[256];
static int g_crc_ready;

EXPORT uint32_t tco_crc32(const uint8_t* data, size_t n)
{
    if (!g_crc_ready) {
        for (uint32_t i = 0; i < 256u; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) { c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1; }
            g_crc_tab[i] = c;
        }
        g_crc_ready = 1;
    }
    uint32_t c = 0xFFFFFFFFu;
    for (size_t i = 0; i < n; ++i) { c = g_crc_tab[(c ^ data[i]) & 0xFFu] ^ (c >> 8); }
    return c ^ 0xFFFFFFFFu;
}

/* ============================ log2 series ============================ */
/* reference: native/src/codec/ctx_ceiling.c:74-89. Compiled with
 * -ffp-contract=off so every operation is a separately rounded IEEE double. */
EXPORT double tco_ctx_log2(double x)
{
    uint64_t bits;
    memcpy(&bits, &x, sizeof(bits));
    const int e = (int)((bits >> 52) & 0x7ffu) - 1023;
    bits = (bits & ~((uint64_t)0x7ff << 52)) | ((uint64_t)1023 << 52);
    double m;
    memcpy(&m, &bits, sizeof(m));
    const double z = (m - 1.0) / (m + 1.0);
    const double z2 = z * z;
    const double at = z * (1.0 + z2 * (1.0 / 3.0 + z2 * (1.0 / 5.0 + z2 * (1.0 / 7.0
                      + z2 * (1.0 / 9.0 + z2 * (1.0 / 11.0 + z2 * (1.0 / 13.0)))))));
    return (double)e + 2.885390081777926814 * at;
}

/* ============================ frame header ============================ */

typedef struct hdr {
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
    /* derived geometry */
    uint16_t pcw[4], pch[4], pvw[4], pvh[4], bcols[4], brows[4];
} hdr;

static int32_t vf(int32_t code, const char* field, unsigned long long v)
{
    return fail(code, "frame header field %s = %llu rejected", field, v);
}

static int32_t vretire(unsigned major)
{
    return fail(TC_ERR_UNSUPPORTED_VERSION, "generation %u retired", major);
}

/* Field rules in table order (frame_header.c:99-535, production build:
 * retired generations are rejected). */
static int32_t hdr_validate(const hdr* h)
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
        } else if (M == 8u) {
            if (!(h->em == 8u && h->cb == 0u && h->cm == 0u)) {
                return vf(TC_ERR_UNSUPPORTED_VERSION, "v8 entropy fields", h->em);
            }
        } else if (M == 9u) {
            if (!(h->em == 9u && h->cb == 0u && h->cm == 0u)) {
                return vf(TC_ERR_UNSUPPORTED_VERSION, "v9 entropy fields", h->em);
            }
        } else if (h->em > 1u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "entropy_mode", h->em);
        }
        if (M == 2u && (h->em == 0u ? h->cb != 0u : h->cb != 1u)) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "codebook_version", h->cb);
        }
        if (M == 2u && h->cm != 0u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "coding_mode", h->cm);
        }
        if ((h->flags & ~0x0003u) != 0u) {
            const uint16_t nb = (uint16_t)(h->flags & 0x000Cu);
            if ((h->flags & ~(0x0003u | 0x000Cu)) != 0u) {
                return vf(TC_ERR_MALFORMED, "v2 flags(reserved bits)", h->flags);
            }
            if (nb != 0u) {
                const int dom = M == 7u && h->em == 7u && h->ftype == 0u &&
                                h->profile == 3u && h->bd == 10u;
                if (!dom) { return vf(TC_ERR_UNSUPPORTED_VERSION, "flags r4/r5 domain", h->flags); }
            }
        }
        if ((h->flags & 0x0002u) != 0u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "tile_layout(V2.0)", h->flags);
        }
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
        const uint8_t tt = h->bd == 12u ? TRAW_LOG0 : 8u;
        if (h->xfer != tt) { return vf(TC_ERR_MALFORMED, "profile(TRAW transfer mismatch for bit depth)", h->xfer); }
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
        if (h->minor == 0u && (h->bd != 10u || h->pf != 0u)) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.2 extended enum in version_minor=0 stream", h->bd);
        }
        if (h->minor == 1u && h->pf != 0u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.3 extended enum in version_minor=1 stream", h->pf);
        }
        if (h->minor == 2u && h->pf > 1u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.4 extended enum in version_minor=2 stream", h->pf);
        }
        if (h->minor < 5u && (h->pf == 3u || h->profile == 7u)) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.6 extended enum in version_minor<5 stream", h->pf);
        }
        if (h->minor < 6u && h->bd == 16u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.7 extended enum in version_minor<6 stream", h->bd);
        }
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
        h->cw > MAX_DIM || h->ch > MAX_DIM) {
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
    if (h->qp > QP_MAX) { return vf(TC_ERR_MALFORMED, "qp_base", h->qp); }
    if (h->qp >= QP_V15_MIN && !((M == 1u && h->minor >= 4u) || M >= 2u)) {
        return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.5 qp>=64 in version_minor<4 stream", h->qp);
    }
    if (h->slices == 0u) { return vf(TC_ERR_MALFORMED, "slice_count(>=1)", h->slices); }
    if (h->slices > MAX_SLICES) { return vf(TC_ERR_LIMIT_EXCEEDED, "slice_count(<=512)", h->slices); }
    if (h->slices < h->planes) { return vf(TC_ERR_MALFORMED, "slice_count(<plane_count)", h->slices); }
    if (h->range > 1u) { return vf(TC_ERR_MALFORMED, "color_range", h->range); }
    if (h->siting > 2u) { return vf(TC_ERR_MALFORMED, "chroma_siting", h->siting); }
    if ((h->pf == 2u || h->pf == 3u) && h->siting != 0u) {
        return vf(TC_ERR_MALFORMED, "chroma_siting(!=0 w/ GBR|CFA)", h->siting);
    }
    switch (h->prim) {
    case 1: case 6: case 9: case 12: break;
    default: return vf(TC_ERR_MALFORMED, "color_primaries(tag)", h->prim);
    }
    switch (h->xfer) {
    case 1: case 8: case 16: case 18: case TRAW_LOG0: break;
    case 13:
        if (M == 1u && h->minor < 7u) {
            return vf(TC_ERR_UNSUPPORTED_VERSION, "v1.8 sRGB transfer(13) in version_minor<7 stream", h->minor);
        }
        break;
    default: return vf(TC_ERR_MALFORMED, "color_transfer(tag)", h->xfer);
    }
    if (h->profile == 7u) {
        const uint8_t tt = h->bd == 16u ? 8u : TRAW_LOG0;
        if (h->xfer != tt) { return vf(TC_ERR_MALFORMED, "color_transfer(profile7 frozen pair)", h->xfer); }
    } else if (h->xfer == TRAW_LOG0) {
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
    if (h->size == 0u || h->size > MAX_PACKET) { return vf(TC_ERR_LIMIT_EXCEEDED, "frame_packet_size(<=256MiB)", h->size); }
    return TC_OK;
}

/* per-plane geometry (frame_header.c:541-588) */
static int32_t hdr_geometry(hdr* h)
{
    if (h->pf == 3u) {
        uint32_t w = ((uint32_t)h->vw + 1u) / 2u, hh = ((uint32_t)h->vh + 1u) / 2u;
        uint32_t cw = (w + 7u) / 8u * 8u, ch = (hh + 7u) / 8u * 8u;
        for (int p = 0; p < 4; ++p) {
            h->pcw[p] = (uint16_t)cw; h->pch[p] = (uint16_t)ch;
            h->pvw[p] = (uint16_t)w; h->pvh[p] = (uint16_t)hh;
            h->bcols[p] = (uint16_t)(cw / 8u); h->brows[p] = (uint16_t)(ch / 8u);
        }
        if (cw > MAX_DIM || ch > MAX_DIM) { return fail(TC_ERR_LIMIT_EXCEEDED, "cfa plane coded dim"); }
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
    if (h->pcw[1] > MAX_DIM || h->pch[1] > MAX_DIM) { return fail(TC_ERR_LIMIT_EXCEEDED, "chroma coded dim"); }
    return TC_OK;
}

static void hdr_pack(const hdr* h, uint8_t o[HDR_SIZE])
{
    o[0] = 'T'; o[1] = 'P'; o[2] = 'I'; o[3] = 'C';
    be16(o + 4, HDR_SIZE);
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
    be32(o + 49, tco_crc32(o, 49u));
}

/* header decode: size, magic, CRC, then fields (frame_header.c:703-781) */
static int32_t hdr_decode(const uint8_t* d, size_t n, hdr* h)
{
    if (n < HDR_SIZE) { return fail(TC_ERR_TRUNCATED, "frame header needs 53 bytes, got %zu", n); }
    if (memcmp(d, "TPIC", 4u) != 0) { return fail(TC_ERR_MALFORMED, "magic mismatch (not TPIC)"); }
    const uint32_t crc = tco_crc32(d, 49u);
    if (ld32(d + 49) != crc) { return fail(TC_ERR_CHECKSUM_MISMATCH, "frame header crc32 mismatch"); }
    memset(h, 0, sizeof(*h));
    if (ld16(d + 4) != HDR_SIZE) { return vf(TC_ERR_MALFORMED, "header_size(!=53)", ld16(d + 4)); }
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
    int32_t rc = hdr_validate(h);
    if (rc != TC_OK) { return rc; }
    return hdr_geometry(h);
}

/* ============================ config -> header ============================ */

/* version_minor selection (codec.c:280-297) */
static void select_minor(hdr* h)
{
    if (h->major >= 2u) { h->minor = 0u; return; }
    h->minor = h->bd == 16u ? 6u : h->pf == 3u ? 5u : h->pf == 2u ? 3u : h->pf == 1u ? 2u
               : h->bd != 10u ? 1u : 0u;
    if (h->qp >= QP_V15_MIN && h->minor < 4u) { h->minor = 4u; }
    if (h->xfer == 13u && h->minor < 7u) { h->minor = 7u; }
}

/* codec.c:299-397 */
static void cfg_to_hdr(const topos_frame_config* c, hdr* h)
{
    memset(h, 0, sizeof(*h));
    h->flags = c->alpha_premultiplied != 0u ? 1u : 0u;
    if ((c->reserved[0] & 0xFFu) == 8u && c->reserved[5] != 0u) {
        h->flags = (uint16_t)(h->flags | ((c->reserved[5] & 1u) ? 0x4u : 0u) |
                              ((c->reserved[5] & 2u) ? 0x8u : 0u));
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
              : (c->pixel_format == 3u ? (c->bit_depth == 16u ? 8u : TRAW_LOG0) : 13u);
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

static uint32_t cfg_slice_rows(const topos_frame_config* c)
{
    return c->slice_rows != 0u ? c->slice_rows : 16u;
}

/* bands per plane (codec.c:405-424) */
static int32_t band_plan(const hdr* h, uint32_t rows_per, uint32_t* total)
{
    uint64_t t = 0;
    for (uint32_t p = 0; p < h->planes; ++p) {
        uint64_t b = ((uint64_t)h->brows[p] + rows_per - 1u) / rows_per;
        t += b == 0u ? 1u : b;
    }
    if (t > MAX_SLICES) { return fail(TC_ERR_LIMIT_EXCEEDED, "slice_rows %u yields %llu slices", rows_per, (unsigned long long)t); }
    if (total) { *total = (uint32_t)t; }
    return TC_OK;
}

/* codec.c:426-605 */
EXPORT int32_t tc_frame_config_validate(const topos_frame_config* c)
{
    if (c == NULL) { return fail(TC_ERR_INVALID_ARGUMENT, "cfg == NULL"); }
    if (c->struct_size != 0u && c->struct_size != sizeof(topos_frame_config)) {
        return fail(TC_ERR_INVALID_ARGUMENT, "cfg struct_size %u", c->struct_size);
    }
    if (c->abi_version != 0u && c->abi_version != TOPOS_CODEC_ABI_VERSION) {
        return fail(TC_ERR_INVALID_ARGUMENT, "cfg abi_version %u unsupported", c->abi_version);
    }
    if (c->visible_width == 0u || c->visible_height == 0u || c->visible_width > MAX_DIM ||
        c->visible_height > MAX_DIM) {
        return fail(TC_ERR_INVALID_ARGUMENT, "visible %ux%u out of 1..16384", c->visible_width, c->visible_height);
    }
    if (c->qp_base > QP_MAX) { return fail(TC_ERR_INVALID_ARGUMENT, "qp_base %u > 95", c->qp_base); }
    if (c->reserved[0] > 11u) { return fail(TC_ERR_INVALID_ARGUMENT, "reserved[0] %u not in {0..11}", c->reserved[0]); }
    if (c->reserved[0] >= 2u && c->reserved[0] <= 7u) {
        return fail(TC_ERR_INVALID_ARGUMENT, "reserved[0] coding selection %u retired", c->reserved[0]);
    }
    if (c->reserved[1] > 1u) { return fail(TC_ERR_INVALID_ARGUMENT, "reserved[1] AQ mode"); }
    if (c->reserved[2] > 1u) { return fail(TC_ERR_INVALID_ARGUMENT, "reserved[2] RDO mode"); }
    {
        const uint8_t em = (uint8_t)(c->reserved[0] & 0xFFu);
        const int end = em >= 10u ? 6 : (em == 9u ? 5 : 3);
        for (int i = end; i < 8; ++i) {
            if (em == 8u && i == 5) { continue; }
            if (c->reserved[i] != 0u) { return fail(TC_ERR_INVALID_ARGUMENT, "reserved[%d] must be 0", i); }
        }
        if (em == 8u && c->reserved[5] != 0u) {
            if ((c->reserved[5] & ~3u) != 0u || c->profile != 3u || c->pixel_format != 0u ||
                c->bit_depth != 10u) {
                return fail(TC_ERR_INVALID_ARGUMENT, "reserved[5] output features require profile 3 / 4:2:2 / 10-bit");
            }
        }
        if (em == 10u || em == 11u) {
            if (c->reserved[3] > 1u) { return fail(TC_ERR_INVALID_ARGUMENT, "temporal frame_type"); }
            const uint32_t want = c->reserved[3] == 0u ? 0u : 1u;
            if (c->reserved[5] != want) { return fail(TC_ERR_INVALID_ARGUMENT, "temporal ref_distance"); }
        }
    }
    if (c->alpha_mode > 2u) { return fail(TC_ERR_INVALID_ARGUMENT, "alpha_mode %u > 2", c->alpha_mode); }
    if (c->alpha_mode == 1u && c->alpha_bit_depth != 16u) {
        return fail(TC_ERR_INVALID_ARGUMENT, "lossless alpha requires bit_depth 16");
    }
    if (c->alpha_mode == 2u && c->alpha_bit_depth != 8u && c->alpha_bit_depth != 10u &&
        c->alpha_bit_depth != 12u) {
        return fail(TC_ERR_INVALID_ARGUMENT, "near-lossless alpha bit_depth %u", c->alpha_bit_depth);
    }
    if (c->pixel_format == 3u) {
        if (c->alpha_mode != 0u) { return fail(TC_ERR_INVALID_ARGUMENT, "TRAW does not support alpha"); }
        if (c->qp_delta_chroma != 0) { return fail(TC_ERR_INVALID_ARGUMENT, "qp_delta_chroma must be 0 for TRAW"); }
    }
    hdr h;
    cfg_to_hdr(c, &h);
    int32_t rc = hdr_geometry(&h);
    if (rc != TC_OK) { return rc; }
    rc = band_plan(&h, cfg_slice_rows(c), NULL);
    if (rc != TC_OK) { return rc; }
    h.slices = (uint16_t)(c->pixel_format == 3u ? 4u : 3u + (c->alpha_mode != 0u ? 1u : 0u));
    h.size = HDR_SIZE;
    rc = hdr_validate(&h);
    if (rc != TC_OK) { return rc; }
    if (c->bit_depth >= 13u && c->reserved[0] != 8u && c->reserved[0] != 9u) {
        return fail(TC_ERR_INVALID_ARGUMENT, "entropy mode %u is 12-bit frozen", c->reserved[0]);
    }
    return TC_OK;
}

/* codec.c:607-647 */
EXPORT size_t tc_frame_packet_bound(const topos_frame_config* c)
{
    if (c == NULL || c->visible_width == 0u || c->visible_height == 0u ||
        c->visible_width > MAX_DIM || c->visible_height > MAX_DIM) {
        return 0u;
    }
    uint64_t cw = (c->visible_width + 7u) / 8u * 8u, ch = (c->visible_height + 7u) / 8u * 8u;
    uint64_t ccw, cch;
    if (c->pixel_format == 0u) {
        ccw = (((uint64_t)c->visible_width + 1u) / 2u + 7u) / 8u * 8u; cch = ch;
    } else if (c->pixel_format == 3u) {
        ccw = (((uint64_t)c->visible_width + 1u) / 2u + 7u) / 8u * 8u;
        cch = (((uint64_t)c->visible_height + 1u) / 2u + 7u) / 8u * 8u;
    } else { ccw = cw; cch = ch; }
    uint64_t blocks = c->pixel_format == 3u ? 4u * ((ccw * cch) / 64u)
                                            : (cw * ch) / 64u + 2u * ((ccw * cch) / 64u);
    uint64_t planes = c->pixel_format == 3u ? 4u : 3u;
    uint64_t bound = 53u + planes * (17u + blocks * 1024u);
    if (c->alpha_mode != 0u) { bound += 17u + cw * ch * 16u; }
    return bound > MAX_PACKET ? (size_t)MAX_PACKET : (size_t)bound;
}

/* ============================ transform / quant ============================ */

/* transform.c:18-67; for wide input (bd > 12) int64 accumulation then the
 * predistortion of transform.c:133-150. */
EXPORT void tco_forward_8x8(const int32_t x[64], int32_t F[64], int wide)
{
    int64_t A[64];
    for (int y = 0; y < 8; ++y) {
        for (int v = 0; v < 8; ++v) {
            int64_t a = 0;
            for (int k = 0; k < 8; ++k) { a += (int64_t)x[y * 8 + k] * TM[v * 8 + k]; }
            A[y * 8 + v] = wide ? a : (int64_t)(int32_t)a;
        }
    }
    for (int u = 0; u < 8; ++u) {
        for (int v = 0; v < 8; ++v) {
            int64_t a = 0;
            for (int y = 0; y < 8; ++y) { a += (int64_t)TM[u * 8 + y] * A[y * 8 + v]; }
            F[u * 8 + v] = (int32_t)a;
        }
    }
    if (wide) {
        for (int i = 0; i < 64; ++i) {
            const int64_t w = TW[i] * (TE[i >> 3] * TE[i & 7]);
            const int64_t num = (int64_t)F[i] * ((int64_t)1 << 32);
            F[i] = num >= 0 ? (int32_t)((2 * num + w) / (2 * w))
                            : -(int32_t)((-2 * num + w) / (2 * w));
        }
    }
}

/* transform.c:69-118 (plain double sum; the reference's symmetric split is an
 * exact regrouping of the same integer sums) */
EXPORT void tco_inverse_8x8(const int32_t coef[64], int32_t xhat[64])
{
    int64_t G[64], B[64];
    for (int i = 0; i < 64; ++i) {
        int32_t c = coef[i];
        if (c > F_MAX_WIDE) { c = F_MAX_WIDE; }
        if (c < -F_MAX_WIDE) { c = -F_MAX_WIDE; }
        G[i] = (int64_t)c * TW[i];
    }
    for (int u = 0; u < 8; ++u) {
        for (int x = 0; x < 8; ++x) {
            int64_t a = 0;
            for (int v = 0; v < 8; ++v) { a += G[u * 8 + v] * TM[v * 8 + x]; }
            B[u * 8 + x] = a;
        }
    }
    for (int y = 0; y < 8; ++y) {
        for (int x = 0; x < 8; ++x) {
            int64_t a = 0;
            for (int u = 0; u < 8; ++u) { a += (int64_t)TM[u * 8 + y] * B[u * 8 + x]; }
            xhat[y * 8 + x] = rshift32_round(a);
        }
    }
}

typedef struct qctx {
    uint32_t Q[64];
    int64_t fclamp;   /* coefficient clamp: 2^25 for bd <= 12, scaled for bd > 12 */
} qctx;

/* quant.c:214-225, 269-308 */
static void qctx_init(qctx* q, const uint16_t qm[64], uint32_t qp, uint8_t bd, uint32_t refined)
{
    for (int i = 0; i < 64; ++i) {
        const uint32_t s = qp_scale(refined, qp);
        uint32_t v = s == 0u ? 0u : (uint32_t)((((uint64_t)qm[i] * s) + 128u) >> 8);
        q->Q[i] = (s != 0u && v == 0u) ? 1u : v;
    }
    q->fclamp = bd > 12u ? ((int64_t)F_MAX * (int64_t)((1u << (bd - 1u)) - 1u)) / 2047 : F_MAX;
}

/* quant.c:310-346: q = sign * (|F| + Q/2 - dz) / Q, dz = Q/4 for AC, 0 for DC */
static void quantize(const qctx* q, const int32_t F[64], int32_t out[64])
{
    for (int i = 0; i < 64; ++i) {
        int64_t v = F[i];
        if (v > q->fclamp) { v = q->fclamp; }
        if (v < -q->fclamp) { v = -q->fclamp; }
        const uint32_t mag = (uint32_t)(v < 0 ? -v : v);
        const uint32_t Q = q->Q[i];
        const uint32_t dz = i == 0 ? 0u : Q / 4u;
        const uint32_t num = mag + (Q >> 1);
        const uint32_t qm = num > dz ? (num - dz) / Q : 0u;
        out[i] = v < 0 ? -(int32_t)qm : (int32_t)qm;
    }
}

/* quant.c:348-357 */
static void dequantize(const qctx* q, const int32_t in[64], int32_t out[64])
{
    for (int i = 0; i < 64; ++i) {
        int64_t v = (int64_t)in[i] * q->Q[i];
        if (v > q->fclamp) { v = q->fclamp; }
        if (v < -q->fclamp) { v = -q->fclamp; }
        out[i] = (int32_t)v;
    }
}

/* ============================ rANS models ============================ */

typedef struct model {
    uint32_t syms;
    uint32_t freq[64];
    uint32_t cum[65];
} model;

/* deterministic normalisation of counts to 4096 (rans.c:10-84) */
static int32_t model_build(model* m, const uint32_t* cnt, uint32_t syms)
{
    memset(m, 0, sizeof(*m));
    uint64_t total = 0;
    for (uint32_t s = 0; s < syms; ++s) { total += cnt[s]; }
    if (total == 0u) { return TC_ERR_INVALID_ARGUMENT; }
    uint32_t f[64], rem[64], sum = 0;
    for (uint32_t s = 0; s < syms; ++s) {
        const uint64_t sc = (uint64_t)cnt[s] * RANS_SCALE;
        f[s] = cnt[s] == 0u ? 0u : (uint32_t)(sc / total);
        rem[s] = (uint32_t)(sc % total);
        if (cnt[s] != 0u && f[s] == 0u) { f[s] = 1u; }
        sum += f[s];
    }
    while (sum > RANS_SCALE) {
        uint32_t big = UINT32_MAX;
        for (uint32_t s = 0; s < syms; ++s) {
            if (f[s] > 1u && (big == UINT32_MAX || f[s] > f[big])) { big = s; }
        }
        if (big == UINT32_MAX) { break; }
        f[big]--; rem[big] = 0u; sum--;
    }
    while (sum < RANS_SCALE) {
        uint32_t best = UINT32_MAX;
        for (uint32_t s = 0; s < syms; ++s) {
            if (cnt[s] == 0u) { continue; }
            if (best == UINT32_MAX || rem[s] > rem[best]) { best = s; }
        }
        if (best == UINT32_MAX) { break; }
        f[best]++; rem[best] = 0u; sum++;
    }
    if (sum != RANS_SCALE) { return TC_ERR_INVALID_ARGUMENT; }
    m->syms = syms;
    uint32_t acc = 0;
    for (uint32_t s = 0; s < syms; ++s) { m->freq[s] = f[s]; m->cum[s] = acc; acc += f[s]; }
    m->cum[syms] = acc;
    return TC_OK;
}

/* proportional 8-bit row bytes (rans.c:283-306) */
static void row_encode(uint8_t* out, uint32_t nsym, const uint32_t* cnt)
{
    uint64_t total = 0;
    for (uint32_t s = 0; s < nsym; ++s) { total += cnt[s]; }
    if (total == 0u) { memset(out, 0, nsym); out[0] = 1u; return; }
    for (uint32_t s = 0; s < nsym; ++s) {
        if (cnt[s] == 0u) { out[s] = 0u; continue; }
        uint64_t v = ((uint64_t)cnt[s] * 255u + total / 2u) / total;
        out[s] = (uint8_t)(v == 0u ? 1u : (v > 255u ? 255u : v));
    }
}

static int32_t row_decode(const uint8_t* in, uint32_t nsym, model* m)
{
    uint32_t c[64];
    for (uint32_t s = 0; s < nsym; ++s) { c[s] = in[s]; }
    return model_build(m, c, nsym);
}

/* context buckets (rans.h:258-283) */
static uint32_t pos_ctx(uint32_t pos) { return pos < 8u ? 0u : pos < 16u ? 1u : pos < 32u ? 2u : 3u; }
static uint32_t prev_ctx(uint32_t cat, int has) { return !has ? 4u : cat == 0u ? 0u : cat == 1u ? 1u : cat <= 3u ? 2u : 3u; }
static uint32_t dcp_ctx(uint32_t cat, int has) { return !has ? 0u : 1u + (cat == 0u ? 0u : cat == 1u ? 1u : cat <= 3u ? 2u : 3u); }

/* candidate cost in bits (codec.c:2159-2175) */
static double rows_cost(const uint32_t* rows, uint32_t nctx, uint32_t nsym)
{
    double bits = 0.0;
    for (uint32_t c = 0; c < nctx; ++c) {
        const uint32_t* cnt = rows + (size_t)c * nsym;
        uint8_t rb[64];
        row_encode(rb, nsym, cnt);
        model m;
        if (row_decode(rb, nsym, &m) != TC_OK) { continue; }
        for (uint32_t s = 0; s < nsym; ++s) {
            if (cnt[s] != 0u) { bits += (double)cnt[s] * (12.0 - tco_ctx_log2((double)m.freq[s])); }
        }
    }
    return bits;
}

/* ============================ rANS encoder ============================ */

typedef struct renc {
    uint32_t x;
    uint8_t* buf;     /* bytes in emission order */
    size_t pos, cap;
} renc;

static void emit_byte(renc* e, uint8_t b)
{
    if (e->pos >= e->cap) {
        size_t nc = e->cap ? e->cap * 2u : 4096u;
        e->buf = (uint8_t*)realloc(e->buf, nc);
        e->cap = nc;
    }
    e->buf[e->pos++] = b;
}

/* symbol put (rans.c:108-133): renormalise then x = (x/f)*4096 + x%f + cum */
static void put_sym(renc* e, uint32_t f, uint32_t cum)
{
    const uint32_t xmax = (RANS_L >> 12 << 8) * f;
    while (e->x >= xmax) { emit_byte(e, (uint8_t)e->x); e->x >>= 8; }
    e->x = ((e->x / f) << 12) + (e->x % f) + cum;
}

/* raw chunk of w bits (rans.h:106-116) */
static void put_chunk(renc* e, uint32_t w, uint32_t c)
{
    const uint32_t thr = 1u << (31u - w);
    while (e->x >= thr) { emit_byte(e, (uint8_t)e->x); e->x >>= 8; }
    e->x = (e->x << w) | (c & ((1u << w) - 1u));
}

/* category suffix: cat-1 magnitude bits, split hi/lo above 23 bits (codec.c:2206-2217) */
static void put_suffix(renc* e, uint32_t cat, uint32_t m)
{
    uint32_t b = cat > 1u ? cat - 1u : 0u;
    if (b == 0u || b > 27u) { return; }
    if (b > 23u) { put_chunk(e, b - 16u, m >> 16); b = 16u; }
    put_chunk(e, b, m);
}

/* ============================ colour slice encode ============================ */

typedef struct band_tok {
    uint32_t blocks, pairs;
    uint32_t* dc_m;
    uint8_t* np;
    uint8_t* run;
    uint32_t* lvl_m;
} band_tok;

/* Token pass for one band (codec.c:1702-1848): forward DCT, quantise, DC
 * residual against the left/top DC of this band, run/level pairs in zigzag
 * order. Returns TC_ERR_INVALID_ARGUMENT on a token-domain violation. */
static int32_t band_tokens(const hdr* h, const uint16_t* coded, uint32_t p, const qctx* q,
                           uint32_t y0, uint32_t bh, band_tok* t,
                           uint32_t dch[DC_SYMS], uint32_t runh[RUN_SYMS], uint32_t lvlh[LVL_SYMS])
{
    const uint32_t cols = h->bcols[p];
    const uint32_t stride = cols * 8u;
    const int32_t mid = (int32_t)(1u << (h->bd - 1u));
    const int wide = h->bd > 12u;
    int32_t* top = (int32_t*)calloc(cols, sizeof(int32_t));
    int32_t* cur = (int32_t*)calloc(cols, sizeof(int32_t));
    int viol = 0;
    uint32_t b = 0, pi = 0;
    for (uint32_t by = 0; by < bh; ++by) {
        for (uint32_t bx = 0; bx < cols; ++bx, ++b) {
            int32_t x[64], F[64], qn[64];
            const uint16_t* src = coded + (size_t)(y0 + by) * 8u * stride + (size_t)bx * 8u;
            for (int yy = 0; yy < 8; ++yy) {
                for (int xx = 0; xx < 8; ++xx) {
                    const int32_t d = (int32_t)src[(size_t)yy * stride + xx] - mid;
                    x[yy * 8 + xx] = wide ? d : (int32_t)(int16_t)d;
                }
            }
            tco_forward_8x8(x, F, wide);
            quantize(q, F, qn);
            const int32_t pred = dc_pred(bx > 0u, bx > 0u ? cur[bx - 1u] : 0, by > 0u, top[bx]);
            uint32_t dcm = map_s(qn[0] - pred);
            if (dcm > M_MAX_DC_BD16) { dcm = M_MAX_DC_BD16; viol = 1; }
            t->dc_m[b] = dcm;
            cur[bx] = qn[0];
            dch[bitlen(dcm)]++;
            uint32_t prev = 0, np = 0;
            for (uint32_t pos = 1; pos < 64u; ++pos) {
                const int32_t v = qn[ZZ[pos]];
                if (v == 0) { continue; }
                uint32_t lm = map_s(v);
                if (lm > M_MAX_LVL_BD16) { lm = M_MAX_LVL_BD16; viol = 1; }
                const uint32_t r = pos - prev - 1u;
                t->run[pi] = (uint8_t)r;
                t->lvl_m[pi] = lm;
                pi++; np++;
                runh[r]++;
                lvlh[bitlen(lm)]++;
                prev = pos;
            }
            t->np[b] = (uint8_t)np;
            runh[63]++;
        }
        int32_t* sw = top; top = cur; cur = sw;
    }
    t->blocks = b;
    t->pairs = pi;
    free(top);
    free(cur);
    if (viol) { return fail(TC_ERR_INVALID_ARGUMENT, "token domain violated"); }
    return TC_OK;
}

/* joint histograms of a token set, added to the rows (codec.c:2116-2151):
 * level by zigzag position, level by the previous level's category in the
 * block, DC category by the previous block's DC category */
static void tok_joints(const band_tok* t, uint32_t jpos[POS_CTX * LVL_SYMS], uint32_t jprev[PREV_CTX * LVL_SYMS],
                       uint32_t jdc[DCP_CTX * DC_SYMS])
{
    size_t pi = 0;
    uint32_t prev_dcc = 0;
    for (uint32_t b = 0; b < t->blocks; ++b) {
        const uint32_t dcc = bitlen(t->dc_m[b]);
        jdc[(b == 0u ? 0u : dcp_ctx(prev_dcc, 1)) * DC_SYMS + dcc]++;
        prev_dcc = dcc;
        uint32_t ppos = 0, pcat = 0;
        for (uint32_t k = 0; k < t->np[b]; ++k, ++pi) {
            const uint32_t cat = bitlen(t->lvl_m[pi]);
            const uint32_t pos = ppos + t->run[pi] + 1u;
            jpos[pos_ctx(pos) * LVL_SYMS + cat]++;
            jprev[prev_ctx(pcat, k != 0u) * LVL_SYMS + cat]++;
            pcat = cat;
            ppos = pos;
        }
    }
}

/* model choice by the candidates' costs in bits, strict < in candidate order
 * (codec.c:2300-2326; the V8 tile choice codec.c:2672-2709 is the same) */
static void pick_models(const uint32_t* dch, const uint32_t* lvlh, const uint32_t* jpos, const uint32_t* jprev,
                        const uint32_t* jdc, uint32_t* lvl_model, uint32_t* dc_model)
{
    uint32_t lm = 0;
    double best = rows_cost(lvlh, 1u, LVL_SYMS) + 8.0 * (double)LVL_SYMS;
    const double pc = rows_cost(jpos, POS_CTX, LVL_SYMS) + 8.0 * (double)(POS_CTX * LVL_SYMS);
    if (pc < best) { best = pc; lm = 1; }
    const double prc = rows_cost(jprev, PREV_CTX, LVL_SYMS) + 8.0 * (double)(PREV_CTX * LVL_SYMS);
    if (prc < best) { lm = 2; }
    const double dn = rows_cost(dch, 1u, DC_SYMS) + 8.0 * (double)DC_SYMS;
    const double dp = rows_cost(jdc, DCP_CTX, DC_SYMS) + 8.0 * (double)(DCP_CTX * DC_SYMS);
    *lvl_model = lm;
    *dc_model = dp < dn ? 1u : 0u;
}

/* backward rANS walk of a token set with given models (codec.c:2410-2492;
 * the V8 segment form codec.c:2528-2640 is the same walk) */
static void tok_stream(const band_tok* t, uint32_t lvl_model, uint32_t dc_model, const model* dcm,
                       const model* rnm, const model* lvm, renc* e)
{
    size_t pi = t->pairs;
    for (uint32_t b = t->blocks; b-- > 0u;) {
        const uint32_t np = t->np[b];
        pi -= np;
        put_sym(e, rnm->freq[63], rnm->cum[63]);
        for (uint32_t k = np; k-- > 0u;) {
            const uint32_t lm = t->lvl_m[pi + k];
            const uint32_t ls = bitlen(lm);
            put_suffix(e, ls, lm);
            uint32_t lc = 0;
            if (lvl_model == 1) {
                uint32_t pos = 0;
                for (uint32_t j = 0; j <= k; ++j) { pos += t->run[pi + j] + 1u; }
                lc = pos_ctx(pos);
            } else if (lvl_model == 2) {
                lc = prev_ctx(k != 0u ? bitlen(t->lvl_m[pi + k - 1u]) : 0u, k != 0u);
            }
            put_sym(e, lvm[lc].freq[ls], lvm[lc].cum[ls]);
            const uint32_t r = t->run[pi + k];
            put_sym(e, rnm->freq[r], rnm->cum[r]);
        }
        const uint32_t dm = t->dc_m[b];
        const uint32_t ds = bitlen(dm);
        put_suffix(e, ds, dm);
        const uint32_t dctx = dc_model == 1 ? dcp_ctx(b != 0u ? bitlen(t->dc_m[b - 1u]) : 0u, b != 0u) : 0u;
        put_sym(e, dcm[dctx].freq[ds], dcm[dctx].cum[ds]);
    }
}

/* stream bytes as the decoder reads them: final state big-endian, then the
 * emitted bytes in reverse (rans.c:165-228) */
static void stream_out(const renc* e, uint8_t* dst)
{
    be32(dst, e->x);
    for (size_t i = 0; i < e->pos; ++i) { dst[4u + i] = e->buf[e->pos - 1u - i]; }
}

/* V7-R2 slice entropy coding (codec.c:2116-2515): joint histograms, per-slice
 * model choice, prefix tables, backward rANS walk, flush. Output payload is
 * appended to *out (malloc'd). */
static int32_t band_rans2(const band_tok* t, const uint32_t dch[DC_SYMS], const uint32_t runh[RUN_SYMS],
                          const uint32_t lvlh[LVL_SYMS], uint8_t** out, size_t* out_n)
{
    uint32_t jpos[POS_CTX * LVL_SYMS] = {0}, jprev[PREV_CTX * LVL_SYMS] = {0}, jdc[DCP_CTX * DC_SYMS] = {0};
    tok_joints(t, jpos, jprev, jdc);
    uint32_t lvl_model, dc_model;
    pick_models(dch, lvlh, jpos, jprev, jdc, &lvl_model, &dc_model);

    const uint32_t nl = lvl_model == 1 ? POS_CTX : lvl_model == 2 ? PREV_CTX : 1u;
    const uint32_t nd = dc_model == 1 ? DCP_CTX : 1u;
    uint8_t prefix[400];
    size_t off = 0;
    prefix[off++] = (uint8_t)(lvl_model | (dc_model << 2));
    model dcm[DCP_CTX], lvm[PREV_CTX], rnm;
    const uint32_t* drows = dc_model == 1 ? jdc : dch;
    for (uint32_t c = 0; c < nd; ++c) {
        row_encode(prefix + off, DC_SYMS, drows + c * DC_SYMS);
        if (row_decode(prefix + off, DC_SYMS, &dcm[c]) != TC_OK) { return TC_ERR_INVALID_ARGUMENT; }
        off += DC_SYMS;
    }
    row_encode(prefix + off, RUN_SYMS, runh);
    if (row_decode(prefix + off, RUN_SYMS, &rnm) != TC_OK) { return TC_ERR_INVALID_ARGUMENT; }
    off += RUN_SYMS;
    const uint32_t* lrows = lvl_model == 1 ? jpos : lvl_model == 2 ? jprev : lvlh;
    for (uint32_t c = 0; c < nl; ++c) {
        row_encode(prefix + off, LVL_SYMS, lrows + c * LVL_SYMS);
        if (row_decode(prefix + off, LVL_SYMS, &lvm[c]) != TC_OK) { return TC_ERR_INVALID_ARGUMENT; }
        off += LVL_SYMS;
    }

    renc e = {RANS_L, NULL, 0, 0};
    tok_stream(t, lvl_model, dc_model, dcm, &rnm, lvm, &e);
    /* payload = prefix | final state (big-endian) | bytes in consumption order */
    const size_t total = off + 4u + e.pos;
    uint8_t* pay = (uint8_t*)malloc(total);
    memcpy(pay, prefix, off);
    stream_out(&e, pay + off);
    free(e.buf);
    *out = pay;
    *out_n = total;
    return TC_OK;
}

/* ============================ bit writer / Rice ============================ */

typedef struct bitw {
    uint8_t* buf;
    size_t n, cap;
    uint64_t acc;
    uint32_t bits;
} bitw;

static void bw_put(bitw* w, uint32_t nbits, uint64_t v)
{
    for (uint32_t i = nbits; i-- > 0u;) {
        w->acc = (w->acc << 1) | ((v >> i) & 1u);
        if (++w->bits == 8u) {
            if (w->n >= w->cap) {
                w->cap = w->cap ? w->cap * 2u : 4096u;
                w->buf = (uint8_t*)realloc(w->buf, w->cap);
            }
            w->buf[w->n++] = (uint8_t)w->acc;
            w->acc = 0;
            w->bits = 0;
        }
    }
}

static void bw_flush(bitw* w)
{
    if (w->bits != 0u) { bw_put(w, 8u - w->bits, 0u); }
}

/* Rice code (rice.h:92-114): q = m >> k; q <= 30: q ones, a zero, k low bits;
 * otherwise 31 ones and the 32-bit literal. */
static void rice_put(bitw* w, uint32_t k, uint32_t m)
{
    const uint32_t q = m >> k;
    if (q <= 30u) {
        for (uint32_t i = 0; i < q; ++i) { bw_put(w, 1u, 1u); }
        bw_put(w, 1u, 0u);
        if (k) { bw_put(w, k, m & ((1u << k) - 1u)); }
    } else {
        bw_put(w, 31u, 0x7FFFFFFFu);
        bw_put(w, 32u, m);
    }
}

typedef struct bitr {
    const uint8_t* d;
    uint64_t nbits, pos;
} bitr;

static int br_bit(bitr* r, uint32_t* b)
{
    if (r->pos >= r->nbits) { return 0; }
    *b = (r->d[r->pos >> 3] >> (7u - (r->pos & 7u))) & 1u;
    r->pos++;
    return 1;
}

static int br_bits(bitr* r, uint32_t n, uint32_t* v)
{
    if (r->nbits - r->pos < n) { return 0; }
    uint32_t a = 0;
    for (uint32_t i = 0; i < n; ++i) { uint32_t b = 0; br_bit(r, &b); a = (a << 1) | b; }
    *v = a;
    return 1;
}

/* Rice decode with domain check (rice.h:153-262): up to 31 leading ones
 * (31 = escape, 32-bit literal follows), then k bits. */
static int32_t rice_get(bitr* r, uint32_t k, uint32_t mmax, uint32_t* m)
{
    uint32_t q = 0, b;
    for (;;) {
        if (q == 31u) { break; }
        if (!br_bit(r, &b)) { return TC_ERR_TRUNCATED; }
        if (b == 0u) { break; }
        q++;
    }
    uint64_t v;
    if (q == 31u) {
        uint32_t lit;
        if (!br_bits(r, 32u, &lit)) { return TC_ERR_TRUNCATED; }
        v = lit;
    } else {
        uint32_t rem = 0;
        if (k && !br_bits(r, k, &rem)) { return TC_ERR_TRUNCATED; }
        v = ((uint64_t)q << k) | rem;
    }
    if (v > mmax) { return TC_ERR_MALFORMED; }
    *m = (uint32_t)v;
    return TC_OK;
}

static uint32_t rice_k(uint64_t sum, uint64_t cnt)
{
    if (cnt == 0u || sum == 0u) { return 0u; }
    const uint64_t mean = sum / cnt;
    uint32_t k = 0;
    while (k < 14u && (mean >> (k + 1u)) != 0u) { ++k; }
    return k;
}

/* ============================ alpha slice encode ============================ */

/* MED residuals of one band + Rice k estimates (codec.c:2969-3010), then
 * run/level pairs with a trailing (run, 0) terminator (block_coding.c:456-481). */
static void alpha_band_encode(const hdr* h, const uint16_t* coded, uint32_t y0, uint32_t bh,
                              uint32_t* k1, uint32_t* k2, uint8_t** out, size_t* out_n)
{
    const uint32_t w = h->pcw[3], rows = bh * 8u, py0 = y0 * 8u;
    int32_t* res = (int32_t*)malloc((size_t)w * rows * sizeof(int32_t));
    uint64_t sl = 0, cl = 0, sr = 0, cr = 0, run = 0;
    for (uint32_t y = 0; y < rows; ++y) {
        const uint16_t* row = coded + (size_t)(py0 + y) * w;
        const uint16_t* up = row - w;
        for (uint32_t x = 0; x < w; ++x) {
            int32_t pred;
            if (y == 0u) { pred = x == 0u ? 0 : row[x - 1u]; }
            else if (x == 0u) { pred = up[0]; }
            else { pred = med(row[x - 1u], up[x], up[x - 1u]); }
            const int32_t r = (int32_t)row[x] - pred;
            res[(size_t)y * w + x] = r;
            if (r != 0) { sr += run; cr++; sl += map_s(r); cl++; run = 0; } else { run++; }
        }
    }
    if (run > 0u) { sr += run; cr++; }
    *k1 = rice_k(sl, cl);
    *k2 = rice_k(sr, cr);
    bitw bw = {0};
    const size_t count = (size_t)w * rows;
    size_t pos = 0;
    uint64_t zr = 0;
    for (size_t i = 0; i < count; ++i) {
        if (res[i] == 0) { zr++; continue; }
        rice_put(&bw, *k2, (uint32_t)zr);
        rice_put(&bw, *k1, map_s(res[i]));
        pos = i + 1u;
        zr = 0;
    }
    if (count - pos > 0u) {
        rice_put(&bw, *k2, (uint32_t)(count - pos));
        rice_put(&bw, *k1, 0u);
    }
    bw_flush(&bw);
    free(res);
    *out = bw.buf;
    *out_n = bw.n;
}

/* ============================ frame encode ============================ */

typedef struct slice_out {
    uint8_t hdr[SH_SIZE];
    uint8_t* payload;
    size_t size;
    int alpha;
} slice_out;

static int32_t v8_encode_frame(const topos_frame_config* cfg, hdr* h, const topos_frame_input* in, uint8_t** pkt_out,
                               size_t* pkt_n, topos_frame_stats* st);

static int32_t encode_frame(const topos_frame_config* cfg, const topos_frame_input* in,
                            uint8_t** pkt_out, size_t* pkt_n, topos_frame_stats* st)
{
    hdr h;
    cfg_to_hdr(cfg, &h);
    int32_t rc = hdr_geometry(&h);
    if (rc != TC_OK) { return rc; }
    const uint32_t srows = cfg_slice_rows(cfg);
    uint32_t total = 0;
    rc = band_plan(&h, srows, &total);
    if (rc != TC_OK) { return rc; }
    h.slices = (uint16_t)total;
    h.size = HDR_SIZE;
    rc = hdr_validate(&h);
    if (rc != TC_OK) { return rc; }
    for (uint32_t p = 0; p < h.planes; ++p) {
        if (in->planes[p] == NULL) { return fail(TC_ERR_INVALID_ARGUMENT, "input plane %u == NULL", p); }
        if (in->strides[p] != 0u && in->strides[p] < h.pvw[p]) {
            return fail(TC_ERR_INVALID_ARGUMENT, "input stride[%u] < visible width", p);
        }
    }
    if (h.major == 8u && h.em == 8u) { return v8_encode_frame(cfg, &h, in, pkt_out, pkt_n, st); }
    if (h.major != 7u || h.em != 7u) {
        return fail(TC_ERR_NOT_IMPLEMENTED, "oracle encodes only the V7-R2 and V8 generations");
    }
    uint16_t qmL[64], qmC[64];
    if (!qm_lookup(h.qm, 0, qmL) || !qm_lookup(h.qm, 1, qmC)) {
        return fail(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id %u", h.qm);
    }
    const uint32_t refined = (h.flags & 0x8u) != 0u;
    slice_out* so = (slice_out*)calloc(total, sizeof(slice_out));
    uint32_t si = 0;
    uint16_t alpha_err = 0;
    for (uint32_t p = 0; p < h.planes && rc == TC_OK; ++p) {
        const uint32_t cw = h.pcw[p], ch = h.pch[p], vw = h.pvw[p], vh = h.pvh[p];
        const size_t sstride = in->strides[p] ? in->strides[p] : vw;
        /* edge-replicate pad to coded size (transform/plane.c:19-41) */
        uint16_t* coded = (uint16_t*)malloc((size_t)cw * ch * sizeof(uint16_t));
        for (uint32_t y = 0; y < ch; ++y) {
            const uint16_t* sr = in->planes[p] + (size_t)(y < vh ? y : vh - 1u) * sstride;
            for (uint32_t x = 0; x < cw; ++x) { coded[(size_t)y * cw + x] = sr[x < vw ? x : vw - 1u]; }
        }
        const int is_alpha = p == 3u && h.amode != 0u;
        if (is_alpha && h.amode == 2u) {
            /* near-lossless alpha pre-quantisation (codec.c:1600-1617) */
            const uint32_t s = 16u - h.abd, half = 1u << (s - 1u), top = (0xFFFFu >> s) << s;
            for (size_t i = 0; i < (size_t)cw * ch; ++i) {
                const uint32_t v = coded[i];
                uint32_t q = ((v + half) >> s) << s;
                if (q > top) { q = top; }
                const uint32_t err = v > q ? v - q : q - v;
                if (err > alpha_err) { alpha_err = (uint16_t)err; }
                coded[i] = (uint16_t)q;
            }
        }
        qctx q;
        int32_t qp_eff = 0;
        if (!is_alpha) {
            const int chroma = h.pf != 3u && (p == 1u || p == 2u);
            const int32_t delta = chroma ? cfg->qp_delta_chroma : cfg->qp_delta_luma;
            int32_t qe = (int32_t)h.qp + delta + (h.bd >= 12u ? 2 * ((int32_t)h.bd - 10) : 0);
            if (qe < 0) { qe = 0; }
            const int32_t ceil = h.qp >= QP_V15_MIN ? (int32_t)QP_MAX : 63;
            if (qe > ceil) { qe = ceil; }
            qp_eff = qe;
            qctx_init(&q, chroma ? qmC : qmL, (uint32_t)qe, h.bd, refined);
        }
        const uint32_t rows = h.brows[p];
        for (uint32_t y0 = 0; y0 < rows && rc == TC_OK; y0 += srows, ++si) {
            const uint32_t bh = rows - y0 < srows ? rows - y0 : srows;
            slice_out* s = &so[si];
            uint8_t* pay = NULL;
            size_t pn = 0;
            uint32_t k1 = 0, k2 = 0, qdb = 64u;
            if (is_alpha) {
                alpha_band_encode(&h, coded, y0, bh, &k1, &k2, &pay, &pn);
                s->alpha = 1;
            } else {
                band_tok t;
                const size_t nb = (size_t)bh * h.bcols[p];
                t.dc_m = (uint32_t*)malloc(nb * sizeof(uint32_t));
                t.np = (uint8_t*)malloc(nb);
                t.run = (uint8_t*)malloc(nb * 63u);
                t.lvl_m = (uint32_t*)malloc(nb * 63u * sizeof(uint32_t));
                uint32_t dch[DC_SYMS] = {0}, runh[RUN_SYMS] = {0}, lvlh[LVL_SYMS] = {0};
                rc = band_tokens(&h, coded, p, &q, y0, bh, &t, dch, runh, lvlh);
                if (rc == TC_OK) { rc = band_rans2(&t, dch, runh, lvlh, &pay, &pn); }
                free(t.dc_m); free(t.np); free(t.run); free(t.lvl_m);
                qdb = (uint32_t)(64 + qp_eff - (int32_t)h.qp);
            }
            if (rc != TC_OK) { break; }
            /* slice header (slice_map.c:7-20) */
            be32(s->hdr, (uint32_t)pn);
            s->hdr[4] = (uint8_t)p;
            be16(s->hdr + 5, y0);
            be16(s->hdr + 7, bh);
            s->hdr[9] = (uint8_t)qdb;
            s->hdr[10] = (uint8_t)k1;
            s->hdr[11] = (uint8_t)k2;
            s->hdr[12] = 0u;
            be32(s->hdr + 13, tco_crc32(pay, pn));
            s->payload = pay;
            s->size = pn;
        }
        free(coded);
    }
    /* assembly: header + slices in plane-major, band-ascending order (codec.c:5660-5693) */
    uint64_t size = HDR_SIZE;
    uint32_t cpay = 0, apay = 0, chdr = 0, ahdr = 0;
    if (rc == TC_OK) {
        for (uint32_t i = 0; i < total; ++i) {
            size += SH_SIZE + so[i].size;
            if (so[i].alpha) { apay += (uint32_t)so[i].size; ahdr += SH_SIZE; }
            else { cpay += (uint32_t)so[i].size; chdr += SH_SIZE; }
        }
        if (size > MAX_PACKET) { rc = fail(TC_ERR_LIMIT_EXCEEDED, "frame packet exceeds 256 MiB"); }
    }
    uint8_t* pkt = NULL;
    if (rc == TC_OK) {
        pkt = (uint8_t*)malloc((size_t)size);
        size_t off = HDR_SIZE;
        for (uint32_t i = 0; i < total; ++i) {
            memcpy(pkt + off, so[i].hdr, SH_SIZE);
            off += SH_SIZE;
            memcpy(pkt + off, so[i].payload, so[i].size);
            off += so[i].size;
        }
        h.size = (uint32_t)size;
        rc = hdr_validate(&h);
        if (rc == TC_OK) { hdr_pack(&h, pkt); }
    }
    for (uint32_t i = 0; i < total; ++i) { free(so[i].payload); }
    free(so);
    if (rc != TC_OK) { free(pkt); return rc; }
    st->packet_size = (uint32_t)size;
    st->color_payload_bytes = cpay;
    st->alpha_payload_bytes = apay;
    st->color_header_bytes = HDR_SIZE + chdr;
    st->alpha_header_bytes = ahdr;
    st->slice_count = (uint16_t)total;
    st->qp_base = h.qp;
    st->alpha_max_abs_error = alpha_err;
    *pkt_out = pkt;
    *pkt_n = (size_t)size;
    return TC_OK;
}

/* ============================ V8 segmented rANS encode ============================ */
/* reference: codec.c:3817-4320 (v8_tokenize_segment, v8_write_table,
 * v8_encode_plane, v8_frame_encode_ready), packet.h:36-82 (layout).
 * Per colour plane: [segment directory S x 12][tile tables T x 350]
 * [segment streams][tile CRCs T x 4]. A segment is sb consecutive blocks in
 * raster order with its own rANS chain; a tile is tile_rows block rows and
 * owns the segments whose first block it holds; its model is chosen from the
 * summed counts of its segments. */
#define V8_EXT 8u
#define V8_TABLE 350u
#define V8_DIR 12u
#define V8_MAXSEG 32u

static uint32_t crc_update(uint32_t crc, const uint8_t* p, size_t n)
{
    (void)tco_crc32(p, 0u);  /* table */
    uint32_t c = crc ^ 0xFFFFFFFFu;
    for (size_t i = 0; i < n; ++i) { c = g_crc_tab[(c ^ p[i]) & 0xFFu] ^ (c >> 8); }
    return c ^ 0xFFFFFFFFu;
}

typedef struct v8tile {
    uint32_t plane, seg_first, seg_count, table_off, stream_off, stream_bytes, crc_stored, crc_ok;
} v8tile;

typedef struct v8view {
    hdr h;
    uint32_t sb, tile_rows;
    uint32_t segs[4], tiles[4], dir_off[4], table_off[4], stream_off[4], crc_off[4];
    uint32_t ntiles;
    v8tile t[MAX_SLICES];
} v8view;

static int32_t v8_scan(const uint8_t* d, size_t n, v8view* v, int verify_crc);

typedef struct v8seg {
    uint32_t dc_m[V8_MAXSEG];
    uint8_t np[V8_MAXSEG];
    uint8_t run[V8_MAXSEG * 63u];
    uint32_t lvl_m[V8_MAXSEG * 63u];
    band_tok t;
} v8seg;

/* tokens of one segment (codec.c:3882-3947): DC predicted inside the segment
 * only (left = the segment's previous block, top = the block one row up when
 * the segment reaches that far), AC run/level pairs in zigzag order */
static int32_t v8_seg_tokens(const int32_t* qplane, uint32_t cols, uint32_t b0, uint32_t nb, v8seg* g,
                             uint32_t dch[DC_SYMS], uint32_t runh[RUN_SYMS], uint32_t lvlh[LVL_SYMS])
{
    int viol = 0;
    uint32_t pi = 0;
    int32_t sdc[V8_MAXSEG];
    for (uint32_t i = 0; i < nb; ++i) {
        const int32_t* q = qplane + (size_t)(b0 + i) * 64u;
        sdc[i] = q[0];
        const int32_t pred = dc_pred(i != 0u, i != 0u ? sdc[i - 1u] : 0, i >= cols, sdc[i >= cols ? i - cols : 0u]);
        uint32_t dcm = map_s(q[0] - pred);
        if (dcm > M_MAX_DC_BD16) { dcm = M_MAX_DC_BD16; viol = 1; }
        g->dc_m[i] = dcm;
        dch[bitlen(dcm)]++;
        uint32_t prev = 0, np = 0;
        for (uint32_t pos = 1; pos < 64u; ++pos) {
            const int32_t v = q[ZZ[pos]];
            if (v == 0) { continue; }
            uint32_t lm = map_s(v);
            if (lm > M_MAX_LVL_BD16) { lm = M_MAX_LVL_BD16; viol = 1; }
            const uint32_t r = pos - prev - 1u;
            g->run[pi] = (uint8_t)r;
            g->lvl_m[pi] = lm;
            pi++; np++;
            runh[r]++;
            lvlh[bitlen(lm)]++;
            prev = pos;
        }
        g->np[i] = (uint8_t)np;
        runh[63]++;
    }
    g->t.blocks = nb;
    g->t.pairs = pi;
    g->t.dc_m = g->dc_m;
    g->t.np = g->np;
    g->t.run = g->run;
    g->t.lvl_m = g->lvl_m;
    if (viol) { return fail(TC_ERR_INVALID_ARGUMENT, "token domain violated (bit_depth 16 qp too low): raise qp"); }
    return TC_OK;
}

/* segments of tile t: [floor(first block / sb), floor(next tile's first block / sb)) */
static void v8_tile_segs(uint32_t t, uint32_t tile_rows, uint32_t cols, uint32_t blocks, uint32_t sb, uint32_t S,
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

/* one colour plane's V8 payload (codec.c:3974-4200) */
static int32_t v8_encode_plane(const hdr* h, uint32_t p, const uint16_t* coded, const qctx* q, uint32_t qdb,
                               uint32_t sb, uint32_t tile_rows, uint8_t** out, size_t* out_n, uint32_t* tiles)
{
    const uint32_t cols = h->bcols[p], rows = h->brows[p], blocks = rows * cols;
    const uint32_t S = (blocks + sb - 1u) / sb;
    const uint32_t T = tile_rows == 0u ? 1u : (rows + tile_rows - 1u) / tile_rows;
    *tiles = T;
    /* quantised coefficients of the whole plane, natural order */
    const uint32_t stride = cols * 8u;
    const int32_t mid = (int32_t)(1u << (h->bd - 1u));
    const int wide = h->bd > 12u;
    int32_t* qp = (int32_t*)malloc((size_t)blocks * 64u * sizeof(int32_t) + 1u);
    for (uint32_t b = 0; b < blocks; ++b) {
        const uint32_t bx = b % cols, by = b / cols;
        int32_t x[64], F[64];
        const uint16_t* src = coded + (size_t)by * 8u * stride + (size_t)bx * 8u;
        for (int yy = 0; yy < 8; ++yy) {
            for (int xx = 0; xx < 8; ++xx) {
                const int32_t d = (int32_t)src[(size_t)yy * stride + xx] - mid;
                x[yy * 8 + xx] = wide ? d : (int32_t)(int16_t)d;
            }
        }
        tco_forward_8x8(x, F, wide);
        quantize(q, F, qp + (size_t)b * 64u);
    }
    uint8_t* dir = (uint8_t*)calloc((size_t)S * V8_DIR + 1u, 1);
    uint8_t* tabs = (uint8_t*)calloc((size_t)T * V8_TABLE, 1);
    uint8_t* streams = NULL;
    size_t slen = 0, scap = 0;
    v8seg* g = (v8seg*)malloc(sizeof(v8seg));
    int32_t rc = TC_OK;
    static const uint32_t zeros[64];
    for (uint32_t t = 0; t < T && rc == TC_OK; ++t) {
        uint32_t sf, sn;
        v8_tile_segs(t, tile_rows, cols, blocks, sb, S, &sf, &sn);
        uint32_t dch[DC_SYMS] = {0}, runh[RUN_SYMS] = {0}, lvlh[LVL_SYMS] = {0};
        uint32_t jpos[POS_CTX * LVL_SYMS] = {0}, jprev[PREV_CTX * LVL_SYMS] = {0}, jdc[DCP_CTX * DC_SYMS] = {0};
        for (uint32_t k = sf; k < sn && rc == TC_OK; ++k) {
            const uint32_t b0 = k * sb, nb = blocks - b0 < sb ? blocks - b0 : sb;
            rc = v8_seg_tokens(qp, cols, b0, nb, g, dch, runh, lvlh);
            if (rc == TC_OK) { tok_joints(&g->t, jpos, jprev, jdc); }
        }
        if (rc != TC_OK) { break; }
        uint32_t lm, dm;
        pick_models(dch, lvlh, jpos, jprev, jdc, &lm, &dm);
        const uint32_t nl = lm == 1 ? POS_CTX : lm == 2 ? PREV_CTX : 1u;
        const uint32_t nd = dm == 1 ? DCP_CTX : 1u;
        const uint32_t* drows = dm == 1 ? jdc : dch;
        const uint32_t* lrows = lm == 1 ? jpos : lm == 2 ? jprev : lvlh;
        /* 350-byte table: flags, 5 DC rows, run row, 5 level rows; rows past the
         * model's contexts hold the all-zero row {1, 0, ...} (codec.c:3949-3971) */
        uint8_t* tb = tabs + (size_t)t * V8_TABLE;
        tb[0] = (uint8_t)(lm | (dm << 2));
        for (uint32_t c = 0; c < DCP_CTX; ++c) { row_encode(tb + 1u + c * DC_SYMS, DC_SYMS, c < nd ? drows + c * DC_SYMS : zeros); }
        row_encode(tb + 1u + DCP_CTX * DC_SYMS, RUN_SYMS, runh);
        for (uint32_t c = 0; c < PREV_CTX; ++c) {
            row_encode(tb + 1u + DCP_CTX * DC_SYMS + RUN_SYMS + c * LVL_SYMS, LVL_SYMS, c < nl ? lrows + c * LVL_SYMS : zeros);
        }
        model dcm[DCP_CTX], lvm[PREV_CTX], rnm;
        for (uint32_t c = 0; c < nd && rc == TC_OK; ++c) {
            if (row_decode(tb + 1u + c * DC_SYMS, DC_SYMS, &dcm[c]) != TC_OK) { rc = TC_ERR_INVALID_ARGUMENT; }
        }
        if (rc == TC_OK && row_decode(tb + 1u + DCP_CTX * DC_SYMS, RUN_SYMS, &rnm) != TC_OK) { rc = TC_ERR_INVALID_ARGUMENT; }
        for (uint32_t c = 0; c < nl && rc == TC_OK; ++c) {
            if (row_decode(tb + 1u + DCP_CTX * DC_SYMS + RUN_SYMS + c * LVL_SYMS, LVL_SYMS, &lvm[c]) != TC_OK) {
                rc = TC_ERR_INVALID_ARGUMENT;
            }
        }
        for (uint32_t k = sf; k < sn && rc == TC_OK; ++k) {
            const uint32_t b0 = k * sb, nb = blocks - b0 < sb ? blocks - b0 : sb;
            uint32_t d0[DC_SYMS] = {0}, r0[RUN_SYMS] = {0}, l0[LVL_SYMS] = {0};
            rc = v8_seg_tokens(qp, cols, b0, nb, g, d0, r0, l0);
            if (rc != TC_OK) { break; }
            renc e = {RANS_L, NULL, 0, 0};
            tok_stream(&g->t, lm, dm, dcm, &rnm, lvm, &e);
            const size_t n = 4u + e.pos;
            if (slen + n > scap) {
                scap = (slen + n) * 2u + 4096u;
                streams = (uint8_t*)realloc(streams, scap);
            }
            stream_out(&e, streams + slen);
            free(e.buf);
            uint8_t* de = dir + (size_t)k * V8_DIR;
            be32(de, (uint32_t)slen);
            be32(de + 4, (uint32_t)n);
            de[8] = (uint8_t)qdb;
            slen += n;
        }
    }
    free(g);
    free(qp);
    if (rc != TC_OK) { free(dir); free(tabs); free(streams); return rc; }
    const size_t total = (size_t)S * V8_DIR + (size_t)T * V8_TABLE + slen + (size_t)T * 4u;
    uint8_t* pay = (uint8_t*)malloc(total + 1u);
    memcpy(pay, dir, (size_t)S * V8_DIR);
    memcpy(pay + (size_t)S * V8_DIR, tabs, (size_t)T * V8_TABLE);
    const size_t sbase = (size_t)S * V8_DIR + (size_t)T * V8_TABLE;
    if (slen) { memcpy(pay + sbase, streams, slen); }
    for (uint32_t t = 0; t < T; ++t) {
        uint32_t sf, sn;
        v8_tile_segs(t, tile_rows, cols, blocks, sb, S, &sf, &sn);
        const uint32_t soff = sf < S ? ld32(dir + (size_t)sf * V8_DIR) : 0u;
        uint32_t sbytes = 0;
        for (uint32_t k = sf; k < sn; ++k) { sbytes += ld32(dir + (size_t)k * V8_DIR + 4u); }
        uint32_t crc = crc_update(0u, tabs + (size_t)t * V8_TABLE, V8_TABLE);
        crc = crc_update(crc, pay + sbase + soff, sbytes);
        be32(pay + sbase + slen + (size_t)t * 4u, crc);
    }
    free(dir);
    free(tabs);
    free(streams);
    *out = pay;
    *out_n = total;
    return TC_OK;
}

/* V8 frame (codec.c:4204-4319): colour planes only; the packet is the frame
 * header (slice count = tiles of all planes), the 8-byte extension
 * (segment blocks log2, tile rows log2, zeros) and the plane payloads */
static int32_t v8_encode_frame(const topos_frame_config* cfg, hdr* h, const topos_frame_input* in, uint8_t** pkt_out,
                               size_t* pkt_n, topos_frame_stats* st)
{
    const uint32_t sb_log2 = cfg->reserved[3] != 0u ? cfg->reserved[3] : 4u;
    const uint32_t tile_log2 = cfg->reserved[4] != 0u ? cfg->reserved[4] : 5u;
    if (sb_log2 < 3u || sb_log2 > 5u) { return fail(TC_ERR_INVALID_ARGUMENT, "v8 reserved[3] sb_log2 %u not in {3,4,5}", sb_log2); }
    if (tile_log2 != 0u && (tile_log2 < 4u || tile_log2 > 6u)) {
        return fail(TC_ERR_INVALID_ARGUMENT, "v8 reserved[4] tile_log2 %u not in {0,4,5,6}", tile_log2);
    }
    if (h->amode != 0u) { return fail(TC_ERR_NOT_IMPLEMENTED, "v8 alpha pending"); }
    if (h->pf == 3u) { return fail(TC_ERR_NOT_IMPLEMENTED, "v8 does not carry CFA (TRAW uses rans2)"); }
    uint16_t qmL[64], qmC[64];
    if (!qm_lookup(h->qm, 0, qmL) || !qm_lookup(h->qm, 1, qmC)) {
        return fail(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id %u", h->qm);
    }
    const uint32_t refined = (h->flags & 0x8u) != 0u;
    uint8_t* pay[3] = {NULL, NULL, NULL};
    size_t pn[3] = {0, 0, 0};
    uint32_t tiles[3] = {0, 0, 0};
    int32_t rc = TC_OK;
    for (uint32_t p = 0; p < 3u && rc == TC_OK; ++p) {
        const uint32_t cw = h->pcw[p], ch = h->pch[p], vw = h->pvw[p], vh = h->pvh[p];
        const size_t sstride = in->strides[p] ? in->strides[p] : vw;
        uint16_t* coded = (uint16_t*)malloc((size_t)cw * ch * sizeof(uint16_t));
        for (uint32_t y = 0; y < ch; ++y) {
            const uint16_t* sr = in->planes[p] + (size_t)(y < vh ? y : vh - 1u) * sstride;
            for (uint32_t x = 0; x < cw; ++x) { coded[(size_t)y * cw + x] = sr[x < vw ? x : vw - 1u]; }
        }
        const int chroma = p == 1u || p == 2u;
        const int32_t delta = chroma ? cfg->qp_delta_chroma : cfg->qp_delta_luma;
        int32_t qe = (int32_t)h->qp + delta + (h->bd >= 12u ? 2 * ((int32_t)h->bd - 10) : 0);
        if (qe < 0) { qe = 0; }
        const int32_t ceil = h->qp >= QP_V15_MIN ? (int32_t)QP_MAX : 63;
        if (qe > ceil) { qe = ceil; }
        qctx q;
        qctx_init(&q, chroma ? qmC : qmL, (uint32_t)qe, h->bd, refined);
        rc = v8_encode_plane(h, p, coded, &q, (uint32_t)(64 + qe - (int32_t)h->qp), 1u << sb_log2,
                             tile_log2 == 0u ? 0u : 1u << tile_log2, &pay[p], &pn[p], &tiles[p]);
        free(coded);
    }
    const uint32_t nt = tiles[0] + tiles[1] + tiles[2];
    if (rc == TC_OK && (nt < 3u || nt > MAX_SLICES)) { rc = fail(TC_ERR_LIMIT_EXCEEDED, "v8 tile count %u out of [3,512]", nt); }
    uint64_t size = HDR_SIZE + V8_EXT;
    for (uint32_t p = 0; p < 3u; ++p) { size += pn[p]; }
    if (rc == TC_OK && size > MAX_PACKET) { rc = fail(TC_ERR_LIMIT_EXCEEDED, "frame packet exceeds 256 MiB"); }
    uint8_t* pkt = NULL;
    if (rc == TC_OK) {
        pkt = (uint8_t*)calloc((size_t)size, 1);
        pkt[HDR_SIZE] = (uint8_t)sb_log2;
        pkt[HDR_SIZE + 1u] = (uint8_t)tile_log2;
        size_t off = HDR_SIZE + V8_EXT;
        for (uint32_t p = 0; p < 3u; ++p) {
            memcpy(pkt + off, pay[p], pn[p]);
            off += pn[p];
        }
        h->slices = (uint16_t)nt;
        h->size = (uint32_t)size;
        rc = hdr_validate(h);
        if (rc == TC_OK) { hdr_pack(h, pkt); }
    }
    for (uint32_t p = 0; p < 3u; ++p) { free(pay[p]); }
    if (rc == TC_OK) {
        /* self-check (codec.c:4289-4304): a structure scan with tile CRCs.
         * It fails where a plane's last segment lies past the last tile's
         * nominal block range (no tile owns it, its directory entry stays
         * zero): the reference rejects such frames as MALFORMED. */
        v8view* v = (v8view*)malloc(sizeof(v8view));
        const int32_t src = v8_scan(pkt, (size_t)size, v, 1);
        if (src != TC_OK) {
            rc = fail(TC_ERR_MALFORMED, "v8 self-check scan failed");
        } else {
            for (uint32_t t = 0; t < v->ntiles; ++t) {
                if (!v->t[t].crc_ok) { rc = fail(TC_ERR_MALFORMED, "v8 self-check: tile %u crc", t); break; }
            }
        }
        free(v);
    }
    if (rc != TC_OK) { free(pkt); return rc; }
    st->packet_size = (uint32_t)size;
    st->color_payload_bytes = (uint32_t)(pn[0] + pn[1] + pn[2]);
    st->alpha_payload_bytes = 0;
    st->color_header_bytes = HDR_SIZE + V8_EXT;
    st->alpha_header_bytes = 0;
    st->slice_count = (uint16_t)nt;
    st->qp_base = h->qp;
    st->alpha_max_abs_error = 0;
    *pkt_out = pkt;
    *pkt_n = (size_t)size;
    return TC_OK;
}

/* codec.c:5970-6018 + 5881-5898 (fixed-QP path; AQ/RDO are out of scope) */
EXPORT int32_t tc_frame_encode(const topos_frame_config* cfg, const topos_frame_input* in,
                               uint8_t* out, size_t out_cap, topos_frame_stats* stats)
{
    topos_frame_stats local;
    memset(&local, 0, sizeof(local));
    if (stats == NULL) { stats = &local; }
    if (cfg != NULL && (cfg->reserved[1] == 1u || cfg->reserved[2] == 1u) && out != NULL) {
        int32_t rc = tc_frame_config_validate(cfg);
        if (rc != TC_OK) { return rc; }
        return fail(TC_ERR_NOT_IMPLEMENTED, "AQ/RDO encode is not implemented");
    }
    stats->struct_size = sizeof(topos_frame_stats);
    stats->abi_version = TOPOS_CODEC_ABI_VERSION;
    if (out == NULL && out_cap != 0u) { return fail(TC_ERR_INVALID_ARGUMENT, "out == NULL with cap %zu", out_cap); }
    int32_t rc = tc_frame_config_validate(cfg);
    if (rc != TC_OK) { return rc; }
    if (in == NULL || (in->struct_size != 0u && in->struct_size != sizeof(topos_frame_input))) {
        return fail(TC_ERR_INVALID_ARGUMENT, "input struct invalid");
    }
    uint8_t* pkt = NULL;
    size_t n = 0;
    rc = encode_frame(cfg, in, &pkt, &n, stats);
    if (rc != TC_OK) { return rc; }
    if (n > out_cap) {
        free(pkt);
        return fail(TC_ERR_BUFFER_TOO_SMALL, "out_cap %zu < %zu bytes needed", out_cap, n);
    }
    if (out != NULL) { memcpy(out, pkt, n); }
    free(pkt);
    return TC_OK;
}

/* ============================ packet parse ============================ */

typedef struct shdr {
    uint32_t size;
    uint8_t plane;
    uint16_t y0, bh;
    uint8_t qdb, k1, k2, k3;
    uint32_t crc;
} shdr;

typedef struct pview {
    hdr h;
    shdr s[MAX_SLICES];
    const uint8_t* pay[MAX_SLICES];
} pview;

/* slice_map.c:48-143 */
static int32_t map_validate(const hdr* h, const shdr* s, uint32_t n)
{
    uint32_t idx = 0;
    for (uint32_t p = 0; p < h->planes; ++p) {
        uint32_t cov = 0;
        const uint32_t rows = h->brows[p];
        while (cov < rows) {
            if (idx >= n) { return fail(TC_ERR_MALFORMED, "plane %u tiling incomplete", p); }
            const shdr* x = &s[idx];
            if (x->plane != p) { return fail(TC_ERR_MALFORMED, "slice %u plane order", idx); }
            if (x->k1 > 14u || x->k2 > 14u || x->k3 > 14u) { return fail(TC_ERR_MALFORMED, "slice %u k > 14", idx); }
            if (h->major == 2u && h->em == 1u && (p < 3u || h->amode == 0u) &&
                (x->k1 > 3u || x->k2 > 3u || x->k3 > 3u)) {
                return fail(TC_ERR_MALFORMED, "slice %u vlc book id > 3", idx);
            }
            if (h->major == 7u && (h->em == 6u || h->em == 7u || h->em == 8u) &&
                (p < 3u || h->amode == 0u) && (x->k1 || x->k2 || x->k3)) {
                return fail(TC_ERR_MALFORMED, "slice %u rans k != 0", idx);
            }
            if (x->y0 != cov) { return fail(TC_ERR_MALFORMED, "slice %u block_y0", idx); }
            if (x->bh == 0u) { return fail(TC_ERR_MALFORMED, "slice %u block_h == 0", idx); }
            if ((uint32_t)x->y0 + x->bh > rows) { return fail(TC_ERR_MALFORMED, "slice %u exceeds plane rows", idx); }
            const int32_t qp = (int32_t)h->qp + (int32_t)x->qdb - 64;
            if (qp < 0 || qp > (int32_t)QP_MAX) { return fail(TC_ERR_MALFORMED, "slice %u effective qp", idx); }
            if (h->amode != 0u && p == 3u && x->k3 != 0u) { return fail(TC_ERR_MALFORMED, "alpha slice k3"); }
            cov += x->bh;
            idx++;
        }
    }
    if (idx != n) { return fail(TC_ERR_MALFORMED, "trailing slices"); }
    return TC_OK;
}

/* packet.c:13-67 */
static int32_t parse_structure(const uint8_t* d, size_t n, pview* v)
{
    memset(v, 0, sizeof(*v));
    int32_t rc = hdr_decode(d, n, &v->h);
    if (rc != TC_OK) { return rc; }
    if (v->h.major == 8u || v->h.major == 9u) {
        return fail(TC_ERR_UNSUPPORTED_VERSION, "v8/v9 packet");
    }
    if ((uint64_t)v->h.size != (uint64_t)n) { return fail(TC_ERR_MALFORMED, "frame_packet_size != actual"); }
    size_t off = HDR_SIZE;
    for (uint32_t i = 0; i < v->h.slices; ++i) {
        if (n - off < SH_SIZE || off > n) { return fail(TC_ERR_TRUNCATED, "slice %u header out of packet", i); }
        const uint8_t* q = d + off;
        shdr* s = &v->s[i];
        s->size = ld32(q); s->plane = q[4]; s->y0 = (uint16_t)ld16(q + 5); s->bh = (uint16_t)ld16(q + 7);
        s->qdb = q[9]; s->k1 = q[10]; s->k2 = q[11]; s->k3 = q[12]; s->crc = ld32(q + 13);
        if (s->k1 > 14u || s->k2 > 14u || s->k3 > 14u) { return fail(TC_ERR_MALFORMED, "slice k > 14"); }
        off += SH_SIZE;
        if ((uint64_t)(n - off) < s->size) { return fail(TC_ERR_TRUNCATED, "slice %u payload out of packet", i); }
        v->pay[i] = d + off;
        off += s->size;
    }
    if (off != n) { return fail(TC_ERR_MALFORMED, "trailing bytes after last slice"); }
    return map_validate(&v->h, v->s, v->h.slices);
}

static void fill_info(const hdr* h, topos_frame_output* o)
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

/* ============================ colour slice decode ============================ */

typedef struct rdec {
    uint32_t x;
    const uint8_t* b;
    size_t n, pos;
} rdec;

static int32_t rd_renorm(rdec* d)
{
    while (d->x < RANS_L) {
        if (d->pos >= d->n) { return TC_ERR_TRUNCATED; }
        d->x = (d->x << 8) | d->b[d->pos++];
    }
    return TC_OK;
}

/* symbol lookup by cumulative frequency (rans.c:249-281 / rans.h:173-186) */
static int32_t rd_sym(rdec* d, const model* m, uint32_t* sym)
{
    const uint32_t slot = d->x & 4095u;
    uint32_t s = 0;
    while (s < m->syms && !(slot >= m->cum[s] && slot < m->cum[s] + m->freq[s])) { ++s; }
    if (s >= m->syms) { return TC_ERR_TRUNCATED; }
    d->x = m->freq[s] * (d->x >> 12) + slot - m->cum[s];
    *sym = s;
    return rd_renorm(d);
}

static int32_t rd_chunk(rdec* d, uint32_t w, uint32_t* c)
{
    *c = d->x & ((1u << w) - 1u);
    d->x >>= w;
    return rd_renorm(d);
}

/* rans.h:160-170, 225-236 */
static int32_t rd_suffix(rdec* d, uint32_t cat, uint32_t* m)
{
    uint32_t v = 0;
    if (cat > 1u) {
        const uint32_t b = cat - 1u;
        int32_t rc;
        if (b > 23u) {
            uint32_t lo, hi;
            if ((rc = rd_chunk(d, 16u, &lo)) != TC_OK) { return rc; }
            if ((rc = rd_chunk(d, b - 16u, &hi)) != TC_OK) { return rc; }
            v = (hi << 16) | lo;
        } else if ((rc = rd_chunk(d, b, &v)) != TC_OK) {
            return rc;
        }
    }
    *m = cat == 0u ? 0u : (1u << (cat - 1u)) | v;
    return TC_OK;
}

typedef struct store {
    uint16_t* dst;
    size_t stride;
    uint32_t vw, vh;
    int32_t mid, maxv;
} store;

/* dequant + inverse + clamp + crop (color_store.h:454-711) */
static void store_block(const store* st, const qctx* q, uint32_t bx, uint32_t by, const int32_t blk[64])
{
    int32_t Fp[64], xh[64];
    dequantize(q, blk, Fp);
    tco_inverse_8x8(Fp, xh);
    const uint32_t px = bx * 8u, py = by * 8u;
    const uint32_t cw = st->vw - px < 8u ? st->vw - px : 8u;
    const uint32_t chh = st->vh - py < 8u ? st->vh - py : 8u;
    for (uint32_t y = 0; y < chh; ++y) {
        for (uint32_t x = 0; x < cw; ++x) {
            int32_t v = xh[y * 8 + x] + st->mid;
            if (v < 0) { v = 0; }
            if (v > st->maxv) { v = st->maxv; }
            st->dst[(size_t)(py + y) * st->stride + px + x] = (uint16_t)v;
        }
    }
}

/* slice_codec.c:554-736 */
static int32_t color_slice_decode(const hdr* h, const shdr* sh, const uint8_t* pay, size_t n,
                                  const qctx* q, const store* st)
{
    if (n < 1u + 121u + 4u) { return TC_ERR_TRUNCATED; }
    const uint8_t flags = pay[0];
    const uint32_t lm = flags & 3u, dm = (flags >> 2) & 1u;
    if ((flags & 0xF8u) != 0u || lm > 2u) { return TC_ERR_MALFORMED; }
    const uint32_t nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u;
    const uint32_t nd = dm == 1u ? DCP_CTX : 1u;
    const size_t prefix = 1u + nd * DC_SYMS + RUN_SYMS + nl * LVL_SYMS;
    if (n < prefix + 4u) { return TC_ERR_TRUNCATED; }
    model dcm[DCP_CTX], lvm[PREV_CTX], rnm;
    size_t off = 1;
    for (uint32_t c = 0; c < nd; ++c, off += DC_SYMS) {
        if (row_decode(pay + off, DC_SYMS, &dcm[c]) != TC_OK) { return TC_ERR_MALFORMED; }
    }
    if (row_decode(pay + off, RUN_SYMS, &rnm) != TC_OK) { return TC_ERR_MALFORMED; }
    off += RUN_SYMS;
    for (uint32_t c = 0; c < nl; ++c, off += LVL_SYMS) {
        if (row_decode(pay + off, LVL_SYMS, &lvm[c]) != TC_OK) { return TC_ERR_MALFORMED; }
    }
    rdec d;
    d.b = pay + prefix;
    d.n = n - prefix;
    d.x = ld32(d.b);
    d.pos = 4u;
    if (d.x < RANS_L) { return TC_ERR_MALFORMED; }
    const uint32_t cols = h->bcols[sh->plane];
    const int wide = h->bd > 12u;
    const uint32_t mdc = wide ? M_MAX_DC_BD16 : M_MAX_DC;
    const uint32_t mlv = wide ? M_MAX_LVL_BD16 : M_MAX_LVL;
    const int64_t dlim = wide ? DC_DOMAIN_BD16 : DC_DOMAIN;
    int32_t* prow = (int32_t*)calloc(cols, sizeof(int32_t));
    int32_t* crow = (int32_t*)calloc(cols, sizeof(int32_t));
    int32_t rc = TC_OK;
    uint32_t prev_dcc = 0;
    int first = 1;
    for (uint32_t by = 0; by < sh->bh && rc == TC_OK; ++by) {
        for (uint32_t bx = 0; bx < cols; ++bx) {
            int32_t blk[64] = {0};
            const model* dmv = &dcm[dm == 1u ? (first ? 0u : dcp_ctx(prev_dcc, 1)) : 0u];
            uint32_t cat, m;
            if ((rc = rd_sym(&d, dmv, &cat)) != TC_OK) { break; }
            if ((rc = rd_suffix(&d, cat, &m)) != TC_OK) { break; }
            if (m > mdc) { rc = TC_ERR_MALFORMED; break; }
            const int32_t pred = dc_pred(bx != 0u, bx != 0u ? crow[bx - 1u] : 0, by != 0u, prow[bx]);
            const int64_t dcv = (int64_t)pred + unmap_s(m);
            if (dcv > dlim || dcv < -dlim) { rc = TC_ERR_MALFORMED; break; }
            blk[0] = (int32_t)dcv;
            prev_dcc = cat;
            first = 0;
            uint32_t pos = 1, pcat = 0;
            int has = 0;
            for (;;) {
                uint32_t r;
                if ((rc = rd_sym(&d, &rnm, &r)) != TC_OK) { break; }
                if (r == 63u) { break; }
                const uint32_t idx = pos + r;
                if (idx > 63u) { rc = TC_ERR_MALFORMED; break; }
                const uint32_t lc = lm == 1u ? pos_ctx(idx) : lm == 2u ? prev_ctx(pcat, has) : 0u;
                if ((rc = rd_sym(&d, &lvm[lc], &cat)) != TC_OK) { break; }
                if ((rc = rd_suffix(&d, cat, &m)) != TC_OK) { break; }
                if (m > mlv) { rc = TC_ERR_MALFORMED; break; }
                blk[ZZ[idx]] = unmap_s(m);
                pcat = cat;
                has = 1;
                pos = idx + 1u;
            }
            if (rc != TC_OK) { break; }
            crow[bx] = blk[0];
            /* natural-order coefficients -> pixels */
            int32_t nat[64];
            memcpy(nat, blk, sizeof(nat));
            store_block(st, q, bx, sh->y0 + by, nat);
        }
        int32_t* sw = prow; prow = crow; crow = sw;
    }
    if (rc == TC_OK && d.pos != d.n) { rc = TC_ERR_MALFORMED; }
    free(prow);
    free(crow);
    return rc;
}

/* ============================ alpha slice decode ============================ */

/* block_coding.c:529-560 + codec.c:7919-7972 + slice_codec.c:1105-1127 */
static int32_t alpha_slice_decode(const hdr* h, const shdr* sh, const uint8_t* pay, size_t n,
                                  uint16_t* dst, size_t stride)
{
    const uint32_t w = h->pcw[3];
    const size_t count = (size_t)w * sh->bh * 8u;
    const uint32_t mask = h->amode == 2u ? ((1u << (16u - h->abd)) - 1u) : 0u;
    const uint32_t y0r = (uint32_t)sh->y0 * 8u;
    uint16_t* prev = (uint16_t*)calloc(w, sizeof(uint16_t));
    uint16_t* cur = (uint16_t*)calloc(w, sizeof(uint16_t));
    bitr r = {pay, (uint64_t)n * 8u, 0};
    int32_t rc = TC_OK;
    size_t pos = 0;
    while (pos < count && rc == TC_OK) {
        const uint64_t remaining = count - pos;
        uint32_t rm, lmv;
        if ((rc = rice_get(&r, sh->k2, (uint32_t)remaining, &rm)) != TC_OK) { break; }
        if ((rc = rice_get(&r, sh->k1, M_MAX_ALPHA, &lmv)) != TC_OK) { break; }
        int32_t level = 0;
        size_t end;
        if (lmv == 0u) {
            if ((uint64_t)rm != remaining) { rc = TC_ERR_MALFORMED; break; }
            end = pos + rm;
        } else {
            if ((uint64_t)rm + 1u > remaining) { rc = TC_ERR_MALFORMED; break; }
            level = unmap_s(lmv);
            end = pos + rm + 1u;
        }
        const size_t at = pos + rm;
        for (size_t i = pos; i < end; ++i) {
            const uint32_t y = (uint32_t)(i / w), x = (uint32_t)(i % w);
            int32_t pred;
            if (y == 0u) { pred = x == 0u ? 0 : cur[x - 1u]; }
            else if (x == 0u) { pred = prev[0]; }
            else { pred = med(cur[x - 1u], prev[x], prev[x - 1u]); }
            int32_t v = pred + (i == at && lmv != 0u ? level : 0);
            if (v < 0) { v = 0; }
            if (v > 65535) { v = 65535; }
            if (mask != 0u && ((uint32_t)v & mask) != 0u) { rc = TC_ERR_MALFORMED; break; }
            cur[x] = (uint16_t)v;
            if (y0r + y < h->pvh[3] && x < h->pvw[3]) { dst[(size_t)(y0r + y) * stride + x] = (uint16_t)v; }
            if (x == w - 1u) { uint16_t* t = prev; prev = cur; cur = t; }
        }
        pos = end;
        if (lmv == 0u) { break; }
    }
    if (rc == TC_OK) {
        /* byte alignment must stay inside the payload, then exact exhaustion */
        uint64_t p = (r.pos + 7u) & ~(uint64_t)7u;
        if (p > r.nbits) { rc = TC_ERR_TRUNCATED; }
        else if (p != r.nbits) { rc = TC_ERR_MALFORMED; }
    }
    free(prev);
    free(cur);
    return rc;
}

/* ============================ deblock ============================ */

static int32_t clip3(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
static uint32_t absu(int32_t v) { return (uint32_t)(v < 0 ? -v : v); }

static int db_gate(int32_t p1, int32_t p0, int32_t q0, int32_t q1, int32_t a, int32_t b)
{
    return absu(q0 - p0) < (uint32_t)a && absu(p1 - p0) < (uint32_t)b && absu(q1 - q0) < (uint32_t)b;
}

static int32_t db_delta(int32_t p1, int32_t p0, int32_t q0, int32_t q1, int32_t clip)
{
    int32_t d = (12 * (q0 - p0) + 4 * (p1 - q1) + 8) >> 4;
    const int32_t dl = q0 - p0;
    const int32_t half = dl >= 0 ? (dl >> 1) : -((-dl) >> 1);
    if (half >= 0) { if (d > half) { d = half; } if (d < 0) { d = 0; } }
    else { if (d < half) { d = half; } if (d > 0) { d = 0; } }
    return clip3(d, -clip, clip);
}

static void db_apply(uint16_t* p1, uint16_t* p0, uint16_t* q0, uint16_t* q1, int32_t d, int32_t maxv)
{
    *p0 = (uint16_t)clip3(*p0 + d, 0, maxv);
    *q0 = (uint16_t)clip3(*q0 - d, 0, maxv);
    const int32_t ds = d >> 1;
    *p1 = (uint16_t)clip3(*p1 + ds, 0, maxv);
    *q1 = (uint16_t)clip3(*q1 - ds, 0, maxv);
}

/* deblock.c:71-341 (full-size delivery, unit 8): vertical edges on every row,
 * then horizontal edges on every boundary row. */
EXPORT void tco_deblock_plane(uint16_t* pix, int32_t stride, uint32_t w, uint32_t h,
                              uint32_t qp, uint32_t table_sel, uint8_t bd)
{
    const uint32_t unit = 8u;
    if (pix == NULL || qp > QP_MAX || w < 2u * unit || h < 2u * unit || (w % unit) || (h % unit)) { return; }
    if (bd < 8u || bd > 16u) { return; }
    const int32_t maxv = (int32_t)((1u << bd) - 1u);
    const uint32_t scale = qp_scale(table_sel, qp);
    uint32_t step = (scale * 3u + 173056u / 2u) / 173056u;
    if (step < 1u) { step = 1u; }
    uint32_t a = step * 2u;
    if (a < 3u) { a = 3u; }
    if (a > 48u) { a = 48u; }
    const int32_t alpha = (int32_t)a, beta = alpha / 2 + 2, clip = alpha >> 1;
    for (uint32_t y = 0; y < h; ++y) {
        uint16_t* row = pix + (size_t)y * stride;
        for (uint32_t x0 = unit; x0 + 1u < w; x0 += unit) {
            const int32_t p1 = row[x0 - 2], p0 = row[x0 - 1], q0 = row[x0], q1 = row[x0 + 1];
            if (db_gate(p1, p0, q0, q1, alpha, beta)) {
                db_apply(row + x0 - 2, row + x0 - 1, row + x0, row + x0 + 1, db_delta(p1, p0, q0, q1, clip), maxv);
            }
        }
    }
    for (uint32_t r = 1; r < h / unit; ++r) {
        const uint32_t y0 = r * unit;
        uint16_t* a2 = pix + (size_t)(y0 - 2u) * stride;
        uint16_t* a1 = pix + (size_t)(y0 - 1u) * stride;
        uint16_t* b0 = pix + (size_t)y0 * stride;
        uint16_t* b1 = pix + (size_t)(y0 + 1u) * stride;
        for (uint32_t x = 0; x < w; ++x) {
            const int32_t p1 = a2[x], p0 = a1[x], q0 = b0[x], q1 = b1[x];
            if (db_gate(p1, p0, q0, q1, alpha, beta)) {
                db_apply(a2 + x, a1 + x, b0 + x, b1 + x, db_delta(p1, p0, q0, q1, clip), maxv);
            }
        }
    }
}

/* ============================ frame decode ============================ */

/* dec_slice_job + dec_frame_finalize (codec.c:8204-8494, 8660-8766) */
static int32_t decode_view(const pview* v, uint16_t* const planes[4], const size_t* strides,
                           topos_frame_output* o)
{
    const hdr* h = &v->h;
    uint16_t qmL[64], qmC[64];
    if (!qm_lookup(h->qm, 0, qmL) || !qm_lookup(h->qm, 1, qmC)) {
        return fail(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id %u", h->qm);
    }
    size_t str[4];
    for (uint32_t p = 0; p < h->planes; ++p) {
        str[p] = (strides && strides[p]) ? strides[p] : h->pvw[p];
        if (str[p] < h->pvw[p]) { return fail(TC_ERR_INVALID_ARGUMENT, "plane %u stride < visible width", p); }
    }
    const uint32_t refined = (h->flags & 0x8u) != 0u;
    uint32_t concealed = 0;
    for (uint32_t i = 0; i < h->slices; ++i) {
        const shdr* sh = &v->s[i];
        const uint32_t p = sh->plane;
        const int is_alpha = p == 3u && h->amode != 0u;
        int32_t rc = TC_OK;
        if (tco_crc32(v->pay[i], sh->size) != sh->crc) {
            rc = TC_ERR_CHECKSUM_MISMATCH;
        } else if (is_alpha) {
            rc = alpha_slice_decode(h, sh, v->pay[i], sh->size, planes[p], str[p]);
        } else {
            const int chroma = h->pf != 3u && (p == 1u || p == 2u);
            qctx q;
            qctx_init(&q, chroma ? qmC : qmL, (uint32_t)((int32_t)h->qp + sh->qdb - 64), h->bd, refined);
            store st = {planes[p], str[p], h->pvw[p], h->pvh[p], (int32_t)(1u << (h->bd - 1u)),
                        (int32_t)((1u << h->bd) - 1u)};
            rc = color_slice_decode(h, sh, v->pay[i], sh->size, &q, &st);
        }
        if (rc != TC_OK) {
            /* conceal the visible rows of the band (codec.c:7975-7985) */
            const uint16_t fill = is_alpha ? 0xFFFFu : (uint16_t)(1u << (h->bd - 1u));
            const uint32_t y0 = (uint32_t)sh->y0 * 8u;
            uint32_t rows = (uint32_t)sh->bh * 8u;
            if (rows > h->pvh[p] - y0) { rows = h->pvh[p] - y0; }
            for (uint32_t y = 0; y < rows; ++y) {
                for (uint32_t x = 0; x < h->pvw[p]; ++x) { planes[p][(size_t)(y0 + y) * str[p] + x] = fill; }
            }
            o->slice_status[i] = TC_FRAME_SLICE_CONCEALED;
            concealed++;
        } else {
            o->slice_status[i] = TC_FRAME_SLICE_OK;
        }
    }
    if ((h->flags & 0x4u) != 0u) {
        for (uint32_t p = 0; p < h->planes && p < 3u; ++p) {
            tco_deblock_plane(planes[p], (int32_t)str[p], h->pvw[p], h->pvh[p], h->qp, refined, h->bd);
        }
    }
    o->concealed_slices = (uint16_t)concealed;
    if (concealed) { fail(TC_WARN_CONCEALED, "%u of %u slices concealed", concealed, h->slices); return TC_WARN_CONCEALED; }
    return TC_OK;
}

/* ============================ V8 segmented rANS decode ============================ */
/* reference: packet.c:103-266 (tc_packet_scan_v8_ex), codec.c:4349-4475
 * (v8_tile_dec_build, v8_decode_segment_q), 4772-4975 (v8_frame_decode).
 * A tile whose CRC (table + member streams) mismatches is concealed whole;
 * a segment whose stream fails is concealed alone; concealment reconstructs
 * the segment's blocks from zero coefficients (the mid level). The call
 * returns TC_OK even when it concealed (concealed_slices and per-tile status
 * tell), and no deblocking runs. */
static int32_t v8_scan(const uint8_t* d, size_t n, v8view* v, int verify_crc)
{
    memset(v, 0, sizeof(*v));
    int32_t rc = hdr_decode(d, n, &v->h);
    if (rc != TC_OK) { return rc; }
    if (v->h.major != 8u && v->h.major != 9u) { return vf(TC_ERR_UNSUPPORTED_VERSION, "version_major(not v8/v9)", v->h.major); }
    if ((uint64_t)v->h.size != (uint64_t)n) { return fail(TC_ERR_MALFORMED, "frame_packet_size %u != actual %zu", v->h.size, n); }
    if (n < HDR_SIZE + V8_EXT) { return fail(TC_ERR_TRUNCATED, "v8 ext header out of packet"); }
    const uint8_t* ext = d + HDR_SIZE;
    if (ext[0] < 3u || ext[0] > 5u) { return vf(TC_ERR_MALFORMED, "segment_blocks_log2", ext[0]); }
    if (ext[1] != 0u && (ext[1] < 4u || ext[1] > 6u)) { return vf(TC_ERR_MALFORMED, "tile_rows_log2", ext[1]); }
    for (uint32_t i = 2; i < V8_EXT; ++i) {
        if (ext[i] != 0u) { return vf(TC_ERR_MALFORMED, "ext reserved(!=0)", ext[i]); }
    }
    v->sb = 1u << ext[0];
    v->tile_rows = ext[1] == 0u ? 0u : 1u << ext[1];
    size_t off = HDR_SIZE + V8_EXT;
    uint32_t nt = 0;
    for (uint32_t p = 0; p < v->h.planes; ++p) {
        const uint32_t rows = v->h.brows[p], cols = v->h.bcols[p], blocks = rows * cols;
        const uint32_t S = (blocks + v->sb - 1u) / v->sb;
        const uint32_t T = (v->tile_rows == 0u || rows == 0u) ? 1u : (rows + v->tile_rows - 1u) / v->tile_rows;
        v->segs[p] = S;
        v->tiles[p] = T;
        v->dir_off[p] = (uint32_t)off;
        if (off > n || (size_t)S * V8_DIR > n - off) { return fail(TC_ERR_TRUNCATED, "v8 plane %u dir out of packet", p); }
        off += (size_t)S * V8_DIR;
        v->table_off[p] = (uint32_t)off;
        if (off > n || (size_t)T * V8_TABLE > n - off) { return fail(TC_ERR_TRUNCATED, "v8 plane %u tables out of packet", p); }
        off += (size_t)T * V8_TABLE;
        v->stream_off[p] = (uint32_t)off;
        const uint8_t* dir = d + v->dir_off[p];
        uint64_t sl = 0;
        for (uint32_t k = 0; k < S; ++k) {
            const uint32_t so = ld32(dir + (size_t)k * V8_DIR), ln = ld32(dir + (size_t)k * V8_DIR + 4u);
            if (ln < 4u) { return vf(TC_ERR_MALFORMED, "segment stream_len(<state)", ln); }
            if (k == 0u) {
                if (so != 0u) { return vf(TC_ERR_MALFORMED, "seg0 stream_off", so); }
            } else if (so != ld32(dir + (size_t)(k - 1u) * V8_DIR) + ld32(dir + (size_t)(k - 1u) * V8_DIR + 4u)) {
                return vf(TC_ERR_MALFORMED, "segment dir gap/off", so);
            }
            sl += ln;
            if (sl > MAX_PACKET) { return vf(TC_ERR_LIMIT_EXCEEDED, "plane stream bytes", sl); }
        }
        if (off > n || sl > n - off) { return fail(TC_ERR_TRUNCATED, "v8 plane %u stream out of packet", p); }
        off += (size_t)sl;
        v->crc_off[p] = (uint32_t)off;
        if (off > n || (size_t)T * 4u > n - off) { return fail(TC_ERR_TRUNCATED, "v8 plane %u crc out of packet", p); }
        for (uint32_t t = 0; t < T; ++t) {
            if (nt + t >= MAX_SLICES) { return vf(TC_ERR_MALFORMED, "slice_count(!= tile total)", nt + t); }
            v8tile* ti = &v->t[nt + t];
            uint32_t sf, sn;
            v8_tile_segs(t, v->tile_rows, cols, blocks, v->sb, S, &sf, &sn);
            ti->plane = p;
            ti->seg_first = sf;
            ti->seg_count = sn - sf;
            ti->table_off = v->table_off[p] + t * V8_TABLE;
        }
        nt += T;
        off += (size_t)T * 4u;
    }
    if (off != n) { return fail(TC_ERR_MALFORMED, "v8 packet has %zu trailing bytes", n - off); }
    if (nt != v->h.slices) { return vf(TC_ERR_MALFORMED, "slice_count(!= tile total)", ((unsigned long long)v->h.slices << 16) | nt); }
    v->ntiles = nt;
    uint32_t tbase = 0;
    for (uint32_t p = 0; p < v->h.planes; ++p) {
        for (uint32_t t = 0; t < v->tiles[p]; ++t) {
            v8tile* ti = &v->t[tbase + t];
            const uint8_t* e0 = d + v->dir_off[p] + (size_t)ti->seg_first * V8_DIR;
            ti->stream_off = ti->seg_count ? v->stream_off[p] + ld32(e0) : v->stream_off[p] + (ti->seg_first < v->segs[p] ? ld32(e0) : 0u);
            ti->stream_bytes = 0;
            for (uint32_t k = 0; k < ti->seg_count; ++k) { ti->stream_bytes += ld32(e0 + (size_t)k * V8_DIR + 4u); }
            ti->crc_stored = ld32(d + v->crc_off[p] + (size_t)t * 4u);
            if (verify_crc) {
                uint32_t crc = crc_update(0u, d + ti->table_off, V8_TABLE);
                crc = crc_update(crc, d + ti->stream_off, ti->stream_bytes);
                ti->crc_ok = crc == ti->crc_stored;
            }
        }
        tbase += v->tiles[p];
    }
    return TC_OK;
}

/* one segment: forward decode with the tile's models, blocks reconstructed
 * into the plane as they decode (codec.c:4382-4475); DC and level magnitudes
 * and the DC domain use the 12-bit limits at every bit depth */
static int32_t v8_segment_decode(const uint8_t* s, size_t n, uint32_t lm, uint32_t dm, const model* dcm,
                                 const model* rnm, const model* lvm, uint32_t nb, uint32_t cols, uint32_t b0,
                                 const qctx* q, const store* st)
{
    if (n < 4u) { return TC_ERR_TRUNCATED; }
    rdec d;
    d.b = s;
    d.n = n;
    d.x = ld32(s);
    d.pos = 4u;
    if (d.x < RANS_L) { return TC_ERR_MALFORMED; }
    int32_t sdc[V8_MAXSEG];
    uint32_t prev_dcc = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        int32_t blk[64] = {0};
        const model* dmv = &dcm[(i == 0u || dm != 1u) ? 0u : dcp_ctx(prev_dcc, 1)];
        uint32_t cat, m;
        int32_t rc;
        if ((rc = rd_sym(&d, dmv, &cat)) != TC_OK) { return rc; }
        if ((rc = rd_suffix(&d, cat, &m)) != TC_OK) { return rc; }
        if (m > M_MAX_DC) { return TC_ERR_MALFORMED; }
        const int32_t pred = dc_pred(i != 0u, i != 0u ? sdc[i - 1u] : 0, i >= cols, sdc[i >= cols ? i - cols : 0u]);
        const int64_t dcv = (int64_t)pred + unmap_s(m);
        if (dcv > DC_DOMAIN || dcv < -DC_DOMAIN) { return TC_ERR_MALFORMED; }
        blk[0] = (int32_t)dcv;
        sdc[i] = blk[0];
        prev_dcc = cat;
        uint32_t pos = 1, pcat = 0;
        int has = 0;
        for (;;) {
            uint32_t r;
            if ((rc = rd_sym(&d, rnm, &r)) != TC_OK) { return rc; }
            if (r == 63u) { break; }
            const uint32_t idx = pos + r;
            if (idx > 63u) { return TC_ERR_MALFORMED; }
            const uint32_t lc = lm == 1u ? pos_ctx(idx) : lm == 2u ? prev_ctx(pcat, has) : 0u;
            if ((rc = rd_sym(&d, &lvm[lc], &cat)) != TC_OK) { return rc; }
            if ((rc = rd_suffix(&d, cat, &m)) != TC_OK) { return rc; }
            if (m > M_MAX_LVL) { return TC_ERR_MALFORMED; }
            blk[ZZ[idx]] = unmap_s(m);
            pcat = cat;
            has = 1;
            pos = idx + 1u;
        }
        const uint32_t ab = b0 + i;
        store_block(st, q, ab % cols, ab / cols, blk);
    }
    return d.pos == d.n ? TC_OK : TC_ERR_MALFORMED;
}

static int32_t v8_decode(const uint8_t* data, size_t size, uint16_t* const planes[4], const size_t* strides,
                         topos_frame_output* o)
{
    v8view* v = (v8view*)malloc(sizeof(v8view));
    int32_t rc = v8_scan(data, size, v, 0);
    if (rc != TC_OK) { free(v); return rc; }
    const hdr* h = &v->h;
    if (h->pf == 3u) { free(v); return fail(TC_ERR_UNSUPPORTED_PIXEL_FORMAT, "v8 does not carry CFA (TRAW uses rans2)"); }
    fill_info(h, o);
    for (uint32_t p = 0; p < h->planes; ++p) {
        if (planes[p] == NULL) { free(v); return fail(TC_ERR_INVALID_ARGUMENT, "v8 planes_out[%u] == NULL", p); }
    }
    /* tile models first: a malformed table rejects the frame */
    typedef struct tmod { uint32_t lm, dm; model dcm[DCP_CTX], rnm, lvm[PREV_CTX]; } tmod;
    tmod* tm = (tmod*)malloc(sizeof(tmod) * (v->ntiles ? v->ntiles : 1u));
    for (uint32_t t = 0; t < v->ntiles && rc == TC_OK; ++t) {
        const uint8_t* tb = data + v->t[t].table_off;
        const uint32_t lm = tb[0] & 3u, dm = (tb[0] >> 2) & 1u;
        if ((tb[0] & 0xF8u) != 0u || lm > 2u) { rc = fail(TC_ERR_MALFORMED, "v8 tile flags %u", tb[0]); break; }
        tm[t].lm = lm;
        tm[t].dm = dm;
        const uint32_t nd = dm ? DCP_CTX : 1u, nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u;
        for (uint32_t c = 0; c < nd && rc == TC_OK; ++c) {
            if (row_decode(tb + 1u + c * DC_SYMS, DC_SYMS, &tm[t].dcm[c]) != TC_OK) { rc = fail(TC_ERR_MALFORMED, "v8 tile dc row %u", c); }
        }
        if (rc == TC_OK && row_decode(tb + 1u + DCP_CTX * DC_SYMS, RUN_SYMS, &tm[t].rnm) != TC_OK) {
            rc = fail(TC_ERR_MALFORMED, "v8 tile run row");
        }
        for (uint32_t c = 0; c < nl && rc == TC_OK; ++c) {
            if (row_decode(tb + 1u + DCP_CTX * DC_SYMS + RUN_SYMS + c * LVL_SYMS, LVL_SYMS, &tm[t].lvm[c]) != TC_OK) {
                rc = fail(TC_ERR_MALFORMED, "v8 tile lvl row %u", c);
            }
        }
    }
    uint16_t qmL[64], qmC[64];
    if (rc == TC_OK && (!qm_lookup(h->qm, 0, qmL) || !qm_lookup(h->qm, 1, qmC))) {
        rc = fail(TC_ERR_UNSUPPORTED_MATRIX, "qmatrix_id %u", h->qm);
    }
    if (rc != TC_OK) { free(tm); free(v); return rc; }
    const uint32_t refined = (h->flags & 0x8u) != 0u;
    uint32_t concealed = 0, tbase = 0;
    for (uint32_t p = 0; p < h->planes; ++p) {
        const size_t str = (strides && strides[p]) ? strides[p] : h->pvw[p];
        const uint32_t cols = h->bcols[p], blocks = h->brows[p] * cols;
        const int chroma = p == 1u || p == 2u;
        store st = {planes[p], str, h->pvw[p], h->pvh[p], (int32_t)(1u << (h->bd - 1u)), (int32_t)((1u << h->bd) - 1u)};
        for (uint32_t t = 0; t < v->tiles[p]; ++t) {
            v8tile* ti = &v->t[tbase + t];
            uint32_t crc = crc_update(0u, data + ti->table_off, V8_TABLE);
            crc = crc_update(crc, data + ti->stream_off, ti->stream_bytes);
            ti->crc_ok = crc == ti->crc_stored;
            uint32_t tile_conc = 0;
            for (uint32_t k = ti->seg_first; k < ti->seg_first + ti->seg_count; ++k) {
                const uint32_t b0 = k * v->sb, nb = blocks - b0 < v->sb ? blocks - b0 : v->sb;
                const uint8_t* de = data + v->dir_off[p] + (size_t)k * V8_DIR;
                int32_t qe = (int32_t)h->qp + (int32_t)de[8] - 64;
                if (qe < 0) { qe = 0; }
                const int32_t ceil = h->qp >= QP_V15_MIN ? (int32_t)QP_MAX : 63;
                if (qe > ceil) { qe = ceil; }
                qctx q;
                qctx_init(&q, chroma ? qmC : qmL, (uint32_t)qe, h->bd, refined);
                int32_t drc = TC_ERR_CHECKSUM_MISMATCH;
                if (ti->crc_ok) {
                    drc = v8_segment_decode(data + v->stream_off[p] + ld32(de), ld32(de + 4u), tm[tbase + t].lm,
                                            tm[tbase + t].dm, tm[tbase + t].dcm, &tm[tbase + t].rnm, tm[tbase + t].lvm,
                                            nb, cols, b0, &q, &st);
                    if (drc != TC_OK) { tile_conc++; }
                }
                if (drc != TC_OK) {
                    static const int32_t zero[64];
                    for (uint32_t i = 0; i < nb; ++i) { store_block(&st, &q, (b0 + i) % cols, (b0 + i) / cols, zero); }
                }
            }
            const int bad = tile_conc != 0u || !ti->crc_ok;
            o->slice_status[tbase + t] = bad ? TC_FRAME_SLICE_CONCEALED : TC_FRAME_SLICE_OK;
            concealed += bad ? 1u : 0u;
        }
        tbase += v->tiles[p];
    }
    o->concealed_slices = (uint16_t)concealed;
    free(tm);
    free(v);
    return TC_OK;
}

/* Generation probe ahead of the V7 structural parse (codec.c:9016-9077):
 * V7-A is retired (UNSUPPORTED_VERSION); V7-B/V8/V9 exist in the reference but
 * are outside this path (NOT_IMPLEMENTED). Returns 0 to continue. */
static int32_t probe_generation(const uint8_t* d, size_t n)
{
    if (n >= HDR_SIZE + 8u && memcmp(d, "TPIC", 4u) == 0 && d[6] == 7u &&
        memcmp(d + HDR_SIZE, "TPLD", 4u) == 0) {
        return fail(TC_ERR_NOT_IMPLEMENTED, "V7-B scalable packets are not implemented");
    }
    if (n > 45u && memcmp(d, "TPIC", 4u) == 0 && d[6] == 7u && d[45] == 5u) {
        return fail(TC_ERR_UNSUPPORTED_VERSION, "generation 7 (V7-A band decode) retired");
    }
    if (n >= HDR_SIZE && memcmp(d, "TPIC", 4u) == 0 && d[6] == 9u) {
        return fail(TC_ERR_NOT_IMPLEMENTED, "V9 packets are not implemented");
    }
    return 0;
}

EXPORT int32_t tc_frame_decode(const uint8_t* data, size_t size, uint16_t* const planes_out[4],
                               const size_t strides[4], topos_frame_output* o)
{
    if (o == NULL) { return fail(TC_ERR_INVALID_ARGUMENT, "out_info == NULL"); }
    memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(topos_frame_output);
    o->abi_version = TOPOS_CODEC_ABI_VERSION;
    if (data == NULL) { return fail(TC_ERR_INVALID_ARGUMENT, "data == NULL"); }
    int32_t rc = probe_generation(data, size);
    if (rc != 0) { return rc; }
    if (size >= HDR_SIZE && memcmp(data, "TPIC", 4u) == 0 && data[6] == 8u) {
        /* V8 (codec.c:9039-9049): query = full scan with tile CRCs + info */
        if (planes_out == NULL) {
            v8view* v8 = (v8view*)malloc(sizeof(v8view));
            rc = v8_scan(data, size, v8, 1);
            if (rc == TC_OK) { fill_info(&v8->h, o); }
            free(v8);
            return rc;
        }
        return v8_decode(data, size, planes_out, strides, o);
    }
    pview* v = (pview*)malloc(sizeof(pview));
    rc = parse_structure(data, size, v);
    if (rc != TC_OK) { free(v); return rc; }
    fill_info(&v->h, o);
    if (planes_out == NULL) { free(v); return TC_OK; }
    if (v->h.major == 7u && v->h.em == 8u && v->h.ftype != 0u) {
        free(v);
        return fail(TC_ERR_STATE, "v7r3 P-frame decode requires a GOP context");
    }
    if (!(v->h.major == 7u && (v->h.em == 7u || v->h.em == 8u))) {
        free(v);
        return fail(TC_ERR_NOT_IMPLEMENTED, "only V7-R2 intra packets are implemented");
    }
    for (uint32_t p = 0; p < v->h.planes; ++p) {
        if (planes_out[p] == NULL) { free(v); return fail(TC_ERR_INVALID_ARGUMENT, "planes_out[%u] == NULL", p); }
    }
    rc = decode_view(v, planes_out, strides, o);
    free(v);
    return rc;
}

/* codec.c:9639-9789: all packets parsed first (any failure rejects the batch),
 * then every frame decoded; return = first non-OK frame status. */
EXPORT int32_t tc_frame_decode_batch(const topos_batch_packet* packets, uint32_t count,
                                     uint16_t* const* planes_out, const size_t* strides,
                                     topos_frame_output* infos)
{
    if (count == 0u) { return TC_OK; }
    if (count > BATCH_MAX) { return fail(TC_ERR_LIMIT_EXCEEDED, "batch count %u", count); }
    if (infos == NULL) { return fail(TC_ERR_INVALID_ARGUMENT, "infos == NULL"); }
    if (packets == NULL) { return fail(TC_ERR_INVALID_ARGUMENT, "batch packets == NULL"); }
    for (uint32_t i = 0; i < count; ++i) {
        if (packets[i].data == NULL) { return fail(TC_ERR_INVALID_ARGUMENT, "packets[%u].data == NULL", i); }
    }
    pview* v = (pview*)malloc(sizeof(pview) * count);
    for (uint32_t i = 0; i < count; ++i) {
        int32_t rc = probe_generation(packets[i].data, packets[i].size);
        if (rc == 0) { rc = parse_structure(packets[i].data, packets[i].size, &v[i]); }
        if (rc != TC_OK) { free(v); return rc; }
    }
    int32_t* frc = (int32_t*)calloc(count, sizeof(int32_t));
    for (uint32_t i = 0; i < count; ++i) {
        topos_frame_output* o = &infos[i];
        memset(o, 0, sizeof(*o));
        o->struct_size = sizeof(topos_frame_output);
        o->abi_version = TOPOS_CODEC_ABI_VERSION;
        fill_info(&v[i].h, o);
        if (planes_out == NULL) { continue; }
        if (v[i].h.major == 7u && v[i].h.em == 8u && v[i].h.ftype != 0u) {
            free(v);
            free(frc);
            return fail(TC_ERR_STATE, "v7r3 P-frame decode requires a GOP context");
        }
        uint16_t* const* pl = planes_out + (size_t)i * 4u;
        for (uint32_t p = 0; p < v[i].h.planes; ++p) {
            if (pl[p] == NULL) { frc[i] = fail(TC_ERR_INVALID_ARGUMENT, "frame %u planes_out[%u] == NULL", i, p); break; }
        }
    }
    if (planes_out == NULL) { free(v); free(frc); return TC_OK; }
    int32_t first = TC_OK;
    for (uint32_t i = 0; i < count; ++i) {
        if (frc[i] == TC_OK) {
            if (!(v[i].h.major == 7u && (v[i].h.em == 7u || v[i].h.em == 8u))) {
                frc[i] = fail(TC_ERR_NOT_IMPLEMENTED, "only V7-R2 intra packets are implemented");
            } else {
                frc[i] = decode_view(&v[i], planes_out + (size_t)i * 4u,
                                     strides ? strides + (size_t)i * 4u : NULL, &infos[i]);
            }
        }
        if (first == TC_OK) { first = frc[i]; }
    }
    free(v);
    free(frc);
    return first;
}

/* codec.c:9807-9831 */
EXPORT int32_t tc_frame_plane_geometry(const topos_frame_output* info, uint32_t plane,
                                       uint32_t* width, uint32_t* height)
{
    if (info == NULL || width == NULL || height == NULL) { return fail(TC_ERR_INVALID_ARGUMENT, "plane geometry args NULL"); }
    if (plane >= info->plane_count) { return fail(TC_ERR_INVALID_ARGUMENT, "plane %u >= plane_count", plane); }
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

EXPORT int32_t tc_abi_version(void) { return TOPOS_CODEC_ABI_VERSION; }
