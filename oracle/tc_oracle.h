/* tc_oracle.h - CPU oracle for the Topos Codec V7-R2 intra frame path.
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is the checker for the GPU library: it
 * is loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
 * never by the product library. It exports the same public frame ABI as the
 * reference (tc_frame_encode / tc_frame_decode / ...) so that the reference's
 * own golden conformance driver can be linked against it, plus a few
 * per-stage hooks (tco_*) used by differential tests.
 */
#ifndef TC_ORACLE_H
#define TC_ORACLE_H

#include "../include/topos_codec.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Exact IEEE-754 log2 series used by the encoder's per-slice model choice
 * (reference: native/src/codec/ctx_ceiling.c:74-89). */
double tco_ctx_log2(double x);

/* Forward 8x8 transform of one block of level-shifted samples.
 * reference: native/src/transform/transform.c:18-67 (+139-150 for bd > 12). */
void tco_forward_8x8(const int32_t x[64], int32_t F[64], int wide);

/* Inverse transform (coefficients already dequantised and clamped).
 * reference: native/src/transform/transform.c:69-118. */
void tco_inverse_8x8(const int32_t coef[64], int32_t xhat[64]);

/* CRC-32 (IEEE, reflected 0xEDB88320). reference: native/src/common/crc32.c */
uint32_t tco_crc32(const uint8_t* data, size_t n);

/* Deblock one plane in place (reference: native/src/codec/deblock.c:71-341). */
void tco_deblock_plane(uint16_t* pix, int32_t stride, uint32_t w, uint32_t h,
                       uint32_t qp, uint32_t table_sel, uint8_t bit_depth);

#ifdef __cplusplus
}
#endif

#endif /* TC_ORACLE_H */
