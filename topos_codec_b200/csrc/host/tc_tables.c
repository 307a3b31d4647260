/* tc_tables.c - frozen bitstream tables and the small table-derived helpers.
 *
 * These constants are part of the bitstream definition, so they must equal the
 * reference's values entry for entry: zigzag scan (reference
 * native/src/entropy/scan.h:12-21), qp scale tables (native/src/transform/quant.c:18-52),
 * quantisation matrices (quant.c:54-186). The CRC-32 polynomial and the
 * log2 series (native/src/codec/ctx_ceiling.c:74-89) are likewise fixed.
 */
#include <string.h>

#include "tc_internal.h"

const uint8_t tc_zigzag[64] = {
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

static const uint32_t k_scale[96] = {
    1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5, 6, 7,
    8, 10, 11, 13, 16, 19, 23, 27, 32, 38, 45, 54, 64, 76, 91, 108,
    128, 152, 181, 215, 256, 304, 362, 431, 512, 609, 724, 861, 1024, 1218, 1448, 1722,
    2048, 2435, 2896, 3444, 4096, 4871, 5793, 6889, 8192, 9742, 11585, 13777, 16384, 19484, 23170, 27555,
    32768, 38968, 46341, 55109, 65536, 77936, 92682, 110218,
    131072, 155872, 185364, 220436, 262144, 311744, 370728, 440872,
    524288, 623487, 741455, 881744, 1048576, 1246974, 1482910, 1763488,
    2097152, 2493948, 2965821, 3526975, 4194304, 4987896, 5931642, 7053950};

/* refined table: identical below qp 64, slower doubling (every 6 qp) above */
static const uint32_t k_scale_refined_hi[32] = {
    32768, 36781, 41285, 46341, 52016, 58386, 65536, 73562,
    82570, 92682, 104032, 116772, 131072, 147123, 165140, 185364,
    208064, 233544, 262144, 294247, 330281, 370728, 416128, 467088,
    524288, 588493, 660561, 741455, 832255, 934175, 1048576, 1176987};

uint32_t tc_qp_scale(uint32_t refined, uint32_t qp)
{
    if (qp > TC_QP_MAX) { return 0u; }
    if (refined != 0u && qp >= 64u) { return k_scale_refined_hi[qp - 64u]; }
    return k_scale[qp];
}

/* id 1: geometric luma/chroma; id 2: 4:4:4 compact; id 3: 4:2:2 low compact;
 * id 4: edge balanced. id 0 is flat 16. */
static const uint16_t k_qm[4][2][64] = {
    {{16, 20, 25, 31, 39, 49, 61, 76, 20, 25, 31, 39, 49, 61, 76, 95,
      25, 31, 39, 49, 61, 76, 95, 119, 31, 39, 49, 61, 76, 95, 119, 149,
      39, 49, 61, 76, 95, 119, 149, 186, 49, 61, 76, 95, 119, 149, 186, 233,
      61, 76, 95, 119, 149, 186, 233, 291, 76, 95, 119, 149, 186, 233, 291, 364},
     {16, 19, 22, 26, 31, 37, 43, 51, 19, 22, 26, 31, 37, 43, 51, 60,
      22, 26, 31, 37, 43, 51, 60, 71, 26, 31, 37, 43, 51, 60, 71, 84,
      31, 37, 43, 51, 60, 71, 84, 99, 37, 43, 51, 60, 71, 84, 99, 117,
      43, 51, 60, 71, 84, 99, 117, 138, 51, 60, 71, 84, 99, 117, 138, 162}},
    {{16, 36, 45, 56, 70, 88, 110, 137, 36, 45, 56, 70, 88, 110, 137, 171,
      45, 56, 70, 88, 110, 137, 171, 214, 56, 70, 88, 110, 137, 171, 214, 268,
      70, 88, 110, 137, 171, 214, 268, 335, 88, 110, 137, 171, 214, 268, 335, 419,
      110, 137, 171, 214, 268, 335, 419, 524, 137, 171, 214, 268, 335, 419, 524, 655},
     {16, 28, 33, 39, 46, 56, 64, 76, 28, 33, 39, 46, 56, 64, 76, 90,
      33, 39, 46, 56, 64, 76, 90, 106, 39, 46, 56, 64, 76, 90, 106, 126,
      46, 56, 64, 76, 90, 106, 126, 148, 56, 64, 76, 90, 106, 126, 148, 176,
      64, 76, 90, 106, 126, 148, 176, 207, 76, 90, 106, 126, 148, 176, 207, 243}},
    {{16, 22, 27, 33, 42, 53, 66, 82, 22, 27, 33, 42, 53, 66, 82, 103,
      27, 33, 42, 53, 66, 82, 103, 129, 33, 42, 53, 66, 82, 103, 129, 161,
      42, 53, 66, 82, 103, 129, 161, 201, 53, 66, 82, 103, 129, 161, 201, 252,
      66, 82, 103, 129, 161, 201, 252, 314, 82, 103, 129, 161, 201, 252, 314, 393},
     {16, 20, 23, 27, 33, 39, 45, 54, 20, 23, 27, 33, 39, 45, 54, 63,
      23, 27, 33, 39, 45, 54, 63, 75, 27, 33, 39, 45, 54, 63, 75, 88,
      33, 39, 45, 54, 63, 75, 88, 104, 39, 45, 54, 63, 75, 88, 104, 123,
      45, 54, 63, 75, 88, 104, 123, 145, 54, 63, 75, 88, 104, 123, 145, 170}},
    {{20, 19, 18, 17, 16, 15, 14, 13, 19, 18, 17, 16, 15, 14, 13, 12,
      18, 17, 16, 15, 14, 13, 12, 11, 17, 16, 15, 14, 13, 12, 11, 11,
      16, 15, 14, 13, 12, 11, 11, 10, 15, 14, 13, 12, 11, 11, 10, 9,
      14, 13, 12, 11, 11, 10, 9, 9, 13, 12, 11, 11, 10, 9, 9, 8},
     {18, 17, 16, 16, 15, 14, 13, 13, 17, 16, 16, 15, 14, 13, 13, 12,
      16, 16, 15, 14, 13, 13, 12, 11, 16, 15, 14, 13, 13, 12, 11, 11,
      15, 14, 13, 13, 12, 11, 11, 10, 14, 13, 13, 12, 11, 11, 10, 10,
      13, 13, 12, 11, 11, 10, 10, 9, 13, 12, 11, 11, 10, 10, 9, 9}}};

int tc_qmatrix(uint8_t id, int chroma, uint16_t out[64])
{
    if (id == 0u) {
        for (int i = 0; i < 64; ++i) { out[i] = 16u; }
        return 1;
    }
    if (id > 4u) { return 0; }
    memcpy(out, k_qm[id - 1u][chroma ? 1 : 0], sizeof(uint16_t) * 64u);
    return 1;
}

/* reference native/src/transform/quant.c:217-225 */
void tc_quant_steps(const uint16_t qm[64], uint32_t qp, uint32_t refined, uint32_t Q[64])
{
    const uint32_t s = tc_qp_scale(refined, qp);
    for (int i = 0; i < 64; ++i) {
        const uint32_t q = s == 0u ? 0u : (uint32_t)((((uint64_t)qm[i] * s) + 128u) >> 8);
        Q[i] = (s != 0u && q == 0u) ? 1u : q;
    }
}

/* coefficient clamp: 2^25 up to 12-bit, scaled by the level-shift range above
 * (reference quant.c:288-294, color_store.h:51-57) */
int64_t tc_coef_clamp(uint8_t bit_depth)
{
    if (bit_depth <= 12u) { return (int64_t)1 << 25; }
    return (((int64_t)1 << 25) * (int64_t)((1u << (bit_depth - 1u)) - 1u)) / 2047;
}

/* The log2 series evaluated with separately rounded IEEE-754 double operations
 * (this file is compiled with -ffp-contract=off). The encoder's model choice
 * only ever takes log2 of an integer frequency in 1..4096, so the device uses
 * this exact table instead of evaluating the series. */
static double series_log2(double x)
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

static double g_log2[4097];
static int g_log2_ready;

const double* tc_log2_table(void)
{
    if (!__atomic_load_n(&g_log2_ready, __ATOMIC_ACQUIRE)) {
        double tmp[4097];
        tmp[0] = 0.0;
        for (int f = 1; f <= 4096; ++f) { tmp[f] = series_log2((double)f); }
        memcpy(g_log2, tmp, sizeof(tmp));
        __atomic_store_n(&g_log2_ready, 1, __ATOMIC_RELEASE);
    }
    return g_log2;
}
