/* tc_crc32.c - host CRC-32 (IEEE 802.3 / zlib, reflected polynomial 0xEDB88320)
 * for frame headers and structural checks; slice payload CRCs run on the GPU.
 * reference: native/src/common/crc32.c */
#include "tc_internal.h"

static uint32_t g_tab[8][256];
static int g_ready;

static void build(void)
{
    for (uint32_t i = 0; i < 256u; ++i) {
        uint32_t c = i;
        for (int k = 0; k < 8; ++k) { c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1; }
        g_tab[0][i] = c;
    }
    for (uint32_t i = 0; i < 256u; ++i) {
        for (int t = 1; t < 8; ++t) { g_tab[t][i] = (g_tab[t - 1][i] >> 8) ^ g_tab[0][g_tab[t - 1][i] & 0xFFu]; }
    }
    __atomic_store_n(&g_ready, 1, __ATOMIC_RELEASE);
}

uint32_t tc_crc32(const uint8_t* d, size_t n)
{
    if (!__atomic_load_n(&g_ready, __ATOMIC_ACQUIRE)) { build(); }
    uint32_t c = 0xFFFFFFFFu;
    while (n >= 8u) {
        const uint32_t a = c ^ ((uint32_t)d[0] | ((uint32_t)d[1] << 8) | ((uint32_t)d[2] << 16) | ((uint32_t)d[3] << 24));
        const uint32_t b = (uint32_t)d[4] | ((uint32_t)d[5] << 8) | ((uint32_t)d[6] << 16) | ((uint32_t)d[7] << 24);
        c = g_tab[7][a & 0xFFu] ^ g_tab[6][(a >> 8) & 0xFFu] ^ g_tab[5][(a >> 16) & 0xFFu] ^ g_tab[4][a >> 24] ^
            g_tab[3][b & 0xFFu] ^ g_tab[2][(b >> 8) & 0xFFu] ^ g_tab[1][(b >> 16) & 0xFFu] ^ g_tab[0][b >> 24];
        d += 8;
        n -= 8u;
    }
    while (n-- > 0u) { c = g_tab[0][(c ^ *d++) & 0xFFu] ^ (c >> 8); }
    return c ^ 0xFFFFFFFFu;
}
