// tcg_decode.cu - V7-R2 intra decode on the GPU (any batch of frames).
//
// Pipeline (one stream):
//   k_dcrc      per slice: CRC-32 of the payload vs the slice header
//                                               (reference codec.c:8204-8225)
//   k_dtables   per colour slice: flags/rows prefix -> rANS models, symbol
//               lookup tables, quantiser steps    (slice_codec.c:554-625)
//   k_dchain    one lane per colour slice, 1-8 slices per warp: serial
//               forward rANS2 decode through bucket tables in shared memory
//               -> zigzag-order coefficients, DC reconstruction, domain
//               checks                          (slice_codec.c:626-736)
//   k_dchain_w  the same decode with one warp per colour slice, the symbol
//               search spread over the lanes (a second tiling; a tuner picks)
//   k_didct     32 blocks per CTA: dequantise, exact inverse transform, clamp, crop
//                                               (color_store.h:529-711)
//   k_dalpha    per alpha slice: Rice run/level decode -> residuals
//                                               (block_coding.c:529-560)
//   k_dalpha_med per alpha slice: MED reconstruction as an anti-diagonal
//               wavefront; near-lossless multiple check (codec.c:7919-7972)
//   k_dconceal  damaged slices: neutral fill of the visible band rows
//                                               (codec.c:7975-7985)
//   k_deblock_v / k_deblock_h  frame-level output filter (deblock.c:71-341)
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "tcg_common.cuh"
#include "tcg_runtime.h"

namespace tcg {

// Per colour slice decode tables (global, built by k_dtables):
//   LUT  11 x 256 u32  per context, bucket b of 16 slots: symbol s0 holding
//                      slot 16b | cum[s0] << 6 | cum[s0+1] << 18
//   CUM  11 x 66 u16   per context: cum[0..nsym], then 4096 up to index 65
//   Q    64 u32        quantiser steps of the slice's effective qp
//   HDR  4 u32         level model, dc model, prefix length
// Context ids: 0..4 DC (by previous DC category), 5 run, 6..10 level.
constexpr uint32_t MAX_CTX = 11u;
constexpr uint32_t LUT_BUCKETS = 256u;
constexpr uint32_t LUT_BYTES = LUT_BUCKETS * 4u;
constexpr uint32_t CUM_LEN = 66u;
constexpr uint32_t CUM_BYTES = CUM_LEN * 2u;
constexpr uint32_t TAB_LUT = 0u;
constexpr uint32_t TAB_CUM = MAX_CTX * LUT_BYTES;
constexpr uint32_t TAB_Q = (TAB_CUM + MAX_CTX * CUM_BYTES + 15u) & ~15u;
constexpr uint32_t TAB_HDR = TAB_Q + 256u;
constexpr uint32_t DTAB_BYTES = TAB_HDR + 16u;

struct DPlane {
    uint64_t out_off;   // element offset in the device output buffer (tight rows)
    uint32_t vis_w, vis_h, coded_w, cols, rows;
    uint32_t bd, kind, alpha_shift, refined;
    uint32_t blk0;
    uint32_t frame;
    uint32_t climit;    // highest zigzag position kept (63 = all)
    uint64_t dst_off;   // delivered plane (the reconstruction itself unless scaled)
    uint32_t dst_w, dst_h;
    uint16_t qm[64];
};

struct DSlice {
    uint32_t frame, plane, pidx, kind;
    uint32_t y0, bh, cols;
    uint32_t blk0, nblk;
    uint32_t size, crc, qp;
    uint32_t k1, k2;
    uint64_t pay;       // payload offset in the device packet buffer
    uint64_t res_off;   // alpha: residual offset (int32 units)
};

struct DFrame {
    uint32_t plane0, planes, bd, deblock, refined, qp_base;
};

// ------------------------------------------------------------------ CRC

__global__ void __launch_bounds__(256) k_dcrc(const DSlice* __restrict__ slices, const uint8_t* __restrict__ pkt,
                                              const uint32_t* __restrict__ crctab, int32_t* __restrict__ status)
{
    __shared__ uint32_t t[8 * 256];
    __shared__ uint32_t scratch[512];
    for (uint32_t i = threadIdx.x; i < 8u * 256u; i += blockDim.x) { t[i] = crctab[i]; }
    __syncthreads();
    const DSlice& S = slices[blockIdx.x];
    const uint32_t c = crc32_block(pkt + S.pay, S.size, t, scratch);
    if (threadIdx.x == 0) { status[blockIdx.x] = c == S.crc ? 0 : TCG_ERR_CHECKSUM_MISMATCH; }
}

// ------------------------------------------------------------------ tables

__global__ void __launch_bounds__(32) k_dtables(const DSlice* __restrict__ slices, const uint32_t* __restrict__ cslices,
                                                const DPlane* __restrict__ planes, const uint8_t* __restrict__ pkt,
                                                const uint32_t* __restrict__ qscale, uint8_t* __restrict__ tabs,
                                                int32_t* __restrict__ status)
{
    __shared__ int32_t bad;
    __shared__ uint32_t meta[3];
    const uint32_t si = cslices[blockIdx.x];
    if (status[si] != 0) { return; }
    const DSlice& S = slices[si];
    const DPlane& P = planes[S.plane];
    const uint8_t* pay = pkt + S.pay;
    uint8_t* tb = tabs + (size_t)blockIdx.x * DTAB_BYTES;
    const uint32_t t = threadIdx.x;
    if (t == 0) {
        bad = 0;
        if (S.size < 1u + 121u + 4u) {
            bad = TCG_ERR_TRUNCATED;
        } else {
            const uint32_t fl = pay[0], lm = fl & 3u, dm = (fl >> 2) & 1u;
            if ((fl & 0xF8u) != 0u || lm > 2u) { bad = TCG_ERR_MALFORMED; }
            const uint32_t nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u, nd = dm ? DCP_CTX : 1u;
            const uint32_t plen = 1u + nd * DC_SYMS + RUN_SYMS + nl * LVL_SYMS;
            if (bad == 0 && S.size < plen + 4u) { bad = TCG_ERR_TRUNCATED; }
            meta[0] = lm; meta[1] = dm; meta[2] = plen;
        }
    }
    __syncwarp();
    if (bad != 0) {
        if (t == 0) { status[si] = bad; }
        return;
    }
    const uint32_t lm = meta[0], dm = meta[1];
    const uint32_t nd = dm ? DCP_CTX : 1u, nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u;
    // one thread per model row, in prefix order: dc rows (contexts 0..nd-1),
    // run (5), level rows (6..6+nl-1)
    const uint32_t nrows = nd + 1u + nl;
    bool ok = true;
    if (t < nrows) {
        uint32_t ctx, off, n;
        if (t < nd) { ctx = t; off = 1u + t * DC_SYMS; n = DC_SYMS; }
        else if (t == nd) { ctx = 5u; off = 1u + nd * DC_SYMS; n = RUN_SYMS; }
        else { ctx = 6u + (t - nd - 1u); off = 1u + nd * DC_SYMS + RUN_SYMS + (t - nd - 1u) * LVL_SYMS; n = LVL_SYMS; }
        uint8_t bytes[64];
        for (uint32_t k = 0; k < n; ++k) { bytes[k] = pay[off + k]; }
        uint16_t fr[64], cu[64];
        ok = model_from_bytes(bytes, n, fr, cu);
        if (ok) {
            uint16_t* cd = reinterpret_cast<uint16_t*>(tb + TAB_CUM + (size_t)ctx * CUM_BYTES);
            for (uint32_t k = 0; k < CUM_LEN; ++k) { cd[k] = k < n ? cu[k] : (uint16_t)4096u; }
            // bucket b (slots 16b..16b+15) records the symbol holding slot 16b:
            // its cumulative start (bits 0-11), index (12-17) and, for symbols
            // 0..24 (the categories whose suffix is at most one 23-bit chunk;
            // 1..24 for levels), frequency (18-30); 0 there sends the chain to
            // its general step
            uint32_t* lut = reinterpret_cast<uint32_t*>(tb + TAB_LUT + (size_t)ctx * LUT_BYTES);
            for (uint32_t sy = 0; sy < n; ++sy) {
                const uint32_t c0 = cu[sy], c1 = c0 + fr[sy];
                const uint32_t ff = (sy <= 24u && (ctx < 6u || sy != 0u)) ? (uint32_t)fr[sy] : 0u;
                for (uint32_t bk = (c0 + 15u) >> 4; bk < LUT_BUCKETS && (bk << 4) < c1; ++bk) {
                    lut[bk] = c0 | (sy << 12) | (ff << 18);
                }
            }
        }
    }
    if (__any_sync(0xFFFFFFFFu, !ok)) {
        if (t == 0) { status[si] = TCG_ERR_MALFORMED; }
        return;
    }
    // quantiser steps for this slice's effective qp
    uint32_t* Q = reinterpret_cast<uint32_t*>(tb + TAB_Q);
    const uint32_t sc = qscale[(P.refined ? 96u : 0u) + S.qp];
    for (uint32_t i = t; i < 64u; i += 32u) {
        const uint32_t q = (uint32_t)((((uint64_t)P.qm[i] * sc) + 128u) >> 8);
        Q[i] = q == 0u ? 1u : q;
    }
    if (t == 0) {
        uint32_t* hdr = reinterpret_cast<uint32_t*>(tb + TAB_HDR);
        hdr[0] = lm; hdr[1] = dm; hdr[2] = meta[2];
    }
}

// ------------------------------------------------------------------ chain
//
// One lane per colour slice; a block holds LANES slices (1, 2, 4 or 8; the
// tuner below picks) and copies their lookup tables into shared memory. A lane's loop iteration decodes one run
// symbol, then either a level (run < 63) or, after an end-of-block run, the
// next block's DC category, and that category's raw suffix: every lane runs
// the same instruction sequence whatever its slice is doing. Symbol lookup is
// one shared-memory read of the bucket holding the slot (16 slots per bucket);
// a slot past the bucket's first symbol walks the cumulative table. Stream
// bytes arrive through a per-lane 64-bit bit window refilled one aligned word
// at a time. Error conditions accumulate in a flag that ends the slice: any
// error conceals it, so only whether one occurred matters, and reading past
// the payload only grows a consumed-byte count that must end equal to the
// payload size.

constexpr uint32_t DCH_LUT_SLOTS = 7u;  // shared-memory bucket tables per slice
constexpr uint32_t DCH_CUM_BYTES = (MAX_CTX * CUM_BYTES + 15u) & ~15u;
constexpr uint32_t DCH_LANE_BYTES = DCH_LUT_SLOTS * LUT_BYTES + DCH_CUM_BYTES;
// block head: the level-context table, three rows of 80 u16 (level models by
// position / by previous category / single), each the offset of a context's
// bucket table in u32 words
constexpr uint32_t DCH_CTX_ROW = 80u;
constexpr uint32_t DCH_HEAD = (3u * DCH_CTX_ROW * 2u + 15u) & ~15u;
__host__ __device__ constexpr uint32_t dch_smem(uint32_t lanes) { return DCH_HEAD + lanes * DCH_LANE_BYTES; }

struct DLane {
    uint32_t x;            // coder state
    uint32_t whi, wlo;     // upcoming stream bits, first bit in the MSB of whi
    uint32_t wbits;        // valid bits in whi:wlo
    uint32_t nxt;          // stream word wi (memory byte order)
    uint32_t wi, wn;       // word index of nxt; words overlapping the payload
    uint32_t wlast;        // last word a load may touch (max(wn, 1) - 1)
    uint32_t a8;           // bit offset of the payload in its first word
    const uint32_t* wb;    // first word of the payload (aligned down)
};

// Predicated global load (a predicate, not a branch) that also asks L2 for
// the 256-byte segment around the word: the stream is read forwards.
__device__ __forceinline__ uint32_t ldg_nc_if(const uint32_t* p, uint32_t old, bool pred)
{
    uint32_t v = old;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q ld.global.nc.L2::256B.u32 %0, [%1];\n\t}"
        : "+r"(v) : "l"(p), "r"((uint32_t)pred));
    return v;
}

// next stream word (a window of 32 bits or fewer takes it below its valid bits)
__device__ __forceinline__ void dl_take_word(DLane& L)
{
    const uint32_t w = __byte_perm(L.nxt, 0u, 0x0123u);
    L.whi |= __funnelshift_rc(w, 0u, L.wbits);  // w >> wbits
    L.wlo |= __funnelshift_rc(0u, w, L.wbits);  // w << (32 - wbits)
    L.wbits += 32u;
    L.wi += 1u;
    L.nxt = ldg_nc_if(L.wb + min(L.wi, L.wlast), L.nxt, true);
}

// keep at least 32 bits in the window: a window of 32 bits or fewer takes the
// next stream word below its valid bits (branch-free; only the load is predicated)
__device__ __forceinline__ void dl_refill(DLane& L)
{
    const bool need = L.wbits <= 32u;
    const uint32_t w = need ? __byte_perm(L.nxt, 0u, 0x0123u) : 0u;
    L.whi |= __funnelshift_rc(w, 0u, L.wbits);  // w >> wbits
    L.wlo |= __funnelshift_rc(0u, w, L.wbits);  // w << (32 - wbits)
    L.wbits += need ? 32u : 0u;
    L.wi += need ? 1u : 0u;
    // past the payload the load repeats its last word: those bits are only
    // consumed by a damaged stream, which the consumed-byte count rejects
    L.nxt = ldg_nc_if(L.wb + min(L.wi, L.wlast), L.nxt, need);
}

// state <- xn followed by the stream bytes that bring it to [2^23, ...): the
// byte count is (leading zeros - 1) / 8, clamped at 0 for states of 2^31 and
// up (xn is never 0 here: a symbol step leaves at least 2^11, a raw chunk at
// least 1). With Refill the window is topped up to 32 bits afterwards; a
// symbol step takes at most 16 bits, so the run symbol, which always follows
// a refilled step, skips it.
template <bool Refill>
__device__ __forceinline__ void dl_renorm(DLane& L, uint32_t xn)
{
    const int32_t lz = __clz((int32_t)xn);
    const uint32_t n8 = (uint32_t)max(lz - 1, 0) & 0x18u;
    L.x = __funnelshift_l(L.whi, xn, n8);
    L.whi = __funnelshift_l(L.wlo, L.whi, n8);
    L.wlo <<= n8;
    L.wbits -= n8;
    if (Refill) { dl_refill(L); }
}

// bytes moved into the state: the first four, then the window's intake minus what it still holds
__device__ __forceinline__ uint32_t dl_consumed(const DLane& L)
{
    return 4u + ((32u - L.a8) + 32u * (L.wi - 2u) - L.wbits) / 8u;
}

__device__ __forceinline__ void dl_init(DLane& L, const uint8_t* b, uint32_t n)
{
    const uintptr_t a = (uintptr_t)b;
    L.wb = reinterpret_cast<const uint32_t*>(a & ~(uintptr_t)3);
    L.wn = (uint32_t)((((a + n + 3u) & ~(uintptr_t)3) - (uintptr_t)L.wb) >> 2);
    L.wlast = L.wn > 0u ? L.wn - 1u : 0u;
    L.a8 = (uint32_t)(a & 3u) * 8u;
    const uint32_t w0 = __byte_perm(__ldg(L.wb), 0u, 0x0123u);
    const uint32_t w1 = 1u < L.wn ? __byte_perm(__ldg(L.wb + 1), 0u, 0x0123u) : 0u;
    L.x = __funnelshift_l(w1, w0, L.a8);  // first four payload bytes, big-endian
    L.whi = w1 << L.a8;
    L.wlo = 0u;
    L.wbits = 32u - L.a8;
    L.wi = 2u;
    L.nxt = __ldg(L.wb + min(2u, L.wlast));
    dl_refill(L);
}

// One symbol: through the bucket table when use_lut, otherwise by walking the
// cumulative table from symbol 0. Both pointers always address valid tables.
template <bool Refill>
__device__ __forceinline__ uint32_t dl_sym(DLane& L, const uint32_t* lut, bool use_lut, const uint16_t* cum)
{
    const uint32_t x = L.x, slot = x & 4095u;
    const uint32_t e = use_lut ? lut[slot >> 4] : 0u;
    uint32_t s = (e >> 12) & 63u, c0 = e & 0xFFFu, c1 = cum[s + 1u];
    while (slot >= c1 && s < CUM_LEN - 2u) {
        ++s;
        c0 = c1;
        c1 = cum[s + 1u];
    }
    dl_renorm<Refill>(L, (c1 - c0) * (x >> 12) + slot - c0);
    return s;
}

// raw chunk of w bits (w <= 23; 0 leaves the state unchanged)
__device__ __forceinline__ uint32_t dl_chunk(DLane& L, uint32_t w)
{
    const uint32_t v = L.x & ~(0xFFFFFFFFu << w);
    dl_renorm<true>(L, L.x >> w);
    return v;
}

// category suffix: m = 2^(cat-1) | (cat-1 raw bits), split 16 + rest above 23
__device__ __forceinline__ uint32_t dl_suffix(DLane& L, uint32_t cat)
{
    const uint32_t b = cat > 1u ? cat - 1u : 0u;
    uint32_t v;
    if (b <= 23u) {
        v = dl_chunk(L, b);
    } else {
        const uint32_t lo = dl_chunk(L, 16u);
        const uint32_t w2 = b - 16u;
        v = (dl_chunk(L, w2 <= 23u ? w2 : 23u) << 16) | lo;
    }
    return cat == 0u ? 0u : (1u << ((cat - 1u) & 31u)) | v;
}

template <uint32_t LANES>
__global__ void __launch_bounds__(32) k_dchain(const DSlice* __restrict__ slices, const uint32_t* __restrict__ order,
                                               uint32_t nc, const uint32_t* __restrict__ slice_tab,
                                               const DPlane* __restrict__ planes, const uint8_t* __restrict__ pkt,
                                               const uint8_t* __restrict__ tabs, int32_t* __restrict__ coef,
                                               int32_t* __restrict__ status)
{
    extern __shared__ __align__(16) uint8_t dsm[];
    uint16_t* ctab = reinterpret_cast<uint16_t*>(dsm);
    const uint32_t t = threadIdx.x;
    // row 1 indexed by the next position (1..64), row 2 by the previous level's
    // category (0..63; index 79 = no previous level in the block), row 0 zero
    for (uint32_t i = t; i < 3u * DCH_CTX_ROW; i += 32u) {
        const uint32_t row = i / DCH_CTX_ROW, k = i % DCH_CTX_ROW;
        const uint32_t ctx = row == 1u ? pos_ctx(k) : (row == 2u ? (k < 64u ? cat_bucket(k) : 4u) : 0u);
        ctab[i] = (uint16_t)(ctx * LUT_BUCKETS);
    }
    // stage every lane's tables: run and level contexts always, DC contexts when they fit
    const uint32_t i0 = blockIdx.x * LANES;
    for (uint32_t l = 0; l < LANES && i0 + l < nc; ++l) {
        const uint32_t sl = order[i0 + l];
        if (status[sl] != 0) { continue; }
        const uint8_t* tb = tabs + (size_t)slice_tab[sl] * DTAB_BYTES;
        const uint32_t* hdr = reinterpret_cast<const uint32_t*>(tb + TAB_HDR);
        const uint32_t lm = hdr[0], dm = hdr[1];
        const uint32_t nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u, nd = dm ? DCP_CTX : 1u;
        const uint32_t ndl = 1u + nl + nd <= DCH_LUT_SLOTS ? nd : 0u;
        uint8_t* ls = dsm + DCH_HEAD + (size_t)l * DCH_LANE_BYTES;
        const uint32_t nlut = 1u + nl + ndl;
        for (uint32_t k = t; k < nlut * (LUT_BYTES / 16u); k += 32u) {
            const uint32_t slot = k / (LUT_BYTES / 16u), part = k % (LUT_BYTES / 16u);
            const uint32_t ctx = slot == 0u ? 5u : (slot <= nl ? 6u + (slot - 1u) : slot - 1u - nl);
            reinterpret_cast<uint4*>(ls + (size_t)slot * LUT_BYTES)[part] =
                reinterpret_cast<const uint4*>(tb + TAB_LUT + (size_t)ctx * LUT_BYTES)[part];
        }
        for (uint32_t k = t; k < DCH_CUM_BYTES / 16u; k += 32u) {
            reinterpret_cast<uint4*>(ls + DCH_LUT_SLOTS * LUT_BYTES)[k] = reinterpret_cast<const uint4*>(tb + TAB_CUM)[k];
        }
    }
    __syncthreads();
    // the lanes with a slice to decode; they stay together until all are done
    const bool live = t < LANES && i0 + t < nc && status[order[i0 + t]] == 0;
    const uint32_t wmask = __ballot_sync(0xFFFFFFFFu, live);
    if (!live) { return; }
    const uint32_t si = order[i0 + t];
    const DSlice& S = slices[si];
    const DPlane& P = planes[S.plane];
    const uint8_t* tb = tabs + (size_t)slice_tab[si] * DTAB_BYTES;
    const uint32_t* hdr = reinterpret_cast<const uint32_t*>(tb + TAB_HDR);
    const uint32_t lm = hdr[0], dm = hdr[1], plen = hdr[2];
    const uint32_t nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u, nd = dm ? DCP_CTX : 1u;
    const bool dc_lut = 1u + nl + nd <= DCH_LUT_SLOTS;
    const uint8_t* ls = dsm + DCH_HEAD + (size_t)t * DCH_LANE_BYTES;
    const uint32_t* lut_run = reinterpret_cast<const uint32_t*>(ls);
    const uint32_t* lut_lvl = lut_run + LUT_BUCKETS;                               // + ctx * LUT_BUCKETS
    const uint32_t* lut_dc = dc_lut ? lut_lvl + nl * LUT_BUCKETS : lut_run;      // + ctx * LUT_BUCKETS when dc_lut
    const uint16_t* cums = reinterpret_cast<const uint16_t*>(ls + DCH_LUT_SLOTS * LUT_BYTES);
    const uint16_t* cum_run = cums + 5u * CUM_LEN;
    const uint16_t* cum_lvl = cums + 6u * CUM_LEN;
    const uint16_t* cum_dc = cums;

    const uint32_t nbytes = S.size - plen;
    DLane L;
    dl_init(L, pkt + S.pay + plen, nbytes);
    uint32_t err = L.x < RANS_L ? 1u : 0u;
    const bool wide = P.bd > 12u;
    const uint32_t mdc = wide ? 0x0FFFFFFFu : 0x08000000u;
    const uint32_t mlv = wide ? 0x07FFFFFFu : 0x04000000u;
    const int64_t dlim = wide ? ((int64_t)1 << 27) : ((int64_t)1 << 25);
    const uint32_t cols = S.cols, nblk = S.nblk;
    int32_t* blk = coef + (size_t)S.blk0 * 64u;

    // first block's DC (no left, no top, context 0)
    uint32_t dcat = dl_sym<true>(L, lut_dc, dc_lut, cum_dc);
    uint32_t m = dl_suffix(L, dcat);
    err |= m > mdc ? 1u : 0u;
    int64_t dcv = unmap_s(m);
    err |= (dcv > dlim || dcv < -dlim) ? 1u : 0u;
    int32_t left = (int32_t)dcv;
    blk[0] = left;
    // DC of the block above the next block, loaded one block ahead of its use
    int32_t top_next = (1u < nblk && 1u >= cols) ? blk[64 - (int64_t)cols * 64] : 0;
    uint32_t prev_dcc = dcat;
    uint32_t b = 0, bx = 0;  // current block within the slice, its column
    uint32_t pos = 1u, pcat = 0u;
    bool has = false;
    // Run symbol 0 covers slots [0, f0) (f0 = 0 when it does not occur). The
    // fast iteration below needs a state below 2^31; a state in [2^23, 2^31)
    // stays there, so only a damaged stream's first state can break that, and
    // such a slice runs the general iteration throughout.
    const bool x_ok = L.x < 0x80000000u;
    const uint32_t f0 = x_ok ? cum_run[1] : 0u;
    // level context (bucket-table offset) of the coefficient at pos if the next
    // run is 0: by position (lm 1), by the previous level's category (lm 2)
    const bool by_pos = lm == 1u;
    const uint16_t* ctl = ctab + (lm == 1u ? 1u : (lm == 2u ? 2u : 0u)) * DCH_CTX_ROW;
    uint32_t lc0 = ctl[by_pos ? 1u : 79u];
    // Lanes of a warp take the same path most of the time; the warp regathers
    // at the top of every iteration (a lane that left for the general step
    // would otherwise run apart from the others until the loop ends), and a
    // finished lane idles until a vote every 8 iterations finds all done. A
    // single lane leaves the loop at once.
#define DCH_FINISH()                                         \
    {                                                        \
        if constexpr (LANES > 1u) { done = true; continue; } \
        else { break; }                                      \
    }
    bool done = false;
    for (uint32_t it = 1u;; ++it) {
        if constexpr (LANES > 1u) {
            __syncwarp(wmask);
            if ((it & 7u) == 0u && __all_sync(wmask, done)) { break; }
            if (done) { continue; }
        }
        // Fast iteration, computed in one straight line and kept only when it
        // applies: run symbol 0 with a state that needs no renormalisation
        // (one multiply-add), then the level at pos from its bucket entry when
        // the slot lies in the bucket's first symbol and the category is 1..24
        // (entries carry frequency 0 otherwise), whose suffix is one chunk of
        // cat-1 <= 23 bits. That chunk's renormalisation count follows from
        // the level step's leading zeros: the state after a step lies in
        // [2^23, 2^31) (1..8 leading zeros) and the chunk adds cat-1.
        const uint32_t x = L.x, slot = x & 4095u;
        const uint32_t x1 = f0 * (x >> 12) + slot;
        const uint32_t slot1 = x1 & 4095u;
        const uint32_t e1 = lut_lvl[lc0 + (slot1 >> 4)];
        // at least 32 bits in the window (a branch: about every other
        // iteration); the fast iteration needs 40 (a level symbol takes up to
        // 16, its suffix up to 24)
        if (L.wbits <= 32u) { dl_take_word(L); }
        const uint32_t c0 = e1 & 0xFFFu, cat = (e1 >> 12) & 63u, fq = e1 >> 18;
        const uint32_t d = slot1 - c0;
        const uint32_t xn = fq * (x1 >> 12) + d;
        const uint32_t lz = (uint32_t)__clz((int32_t)xn);
        const uint32_t n8 = (lz - 1u) & 0x18u;
        const uint32_t x2 = __funnelshift_l(L.whi, xn, n8);
        const uint32_t whi2 = __funnelshift_l(L.wlo, L.whi, n8);
        const uint32_t wlo2 = L.wlo << n8;
        const uint32_t bw = (cat - 1u) & 31u, hb = 1u << bw;
        const uint32_t mm = (x2 & (hb - 1u)) | hb;
        const uint32_t n8s = (lz - n8 + bw - 1u) & 0x18u;
        if (slot < f0 && x1 >= RANS_L && pos < 64u && L.wbits >= 40u && d < fq) {
            L.x = __funnelshift_l(whi2, x2 >> bw, n8s);
            L.whi = __funnelshift_l(wlo2, whi2, n8s);
            L.wlo = wlo2 << n8s;
            L.wbits -= n8 + n8s;
            blk[pos] = (int32_t)mm;
            ++pos;
            pcat = cat;
            has = true;
            lc0 = ctl[by_pos ? pos : cat];
            continue;
        }
        if (err != 0u) { DCH_FINISH(); }
        // general iteration: any run symbol, end of block and the next block's DC
        const uint32_t r = dl_sym<false>(L, lut_run, true, cum_run);
        const bool geob = r == 63u;
        const uint32_t idx = pos + r;
        if (!geob && idx > 63u) {
            err = 1u;
            DCH_FINISH();
        }
        if (geob && b + 1u >= nblk) { DCH_FINISH(); }  // last block done
        // second symbol: the level (context by position or previous level) or the next block's DC
        const uint32_t lc = lm == 1u ? pos_ctx(idx & 63u) : (lm == 2u ? prev_ctx(pcat, has) : 0u);
        const uint32_t dctx = dm ? dcp_ctx(prev_dcc, true) : 0u;
        const uint32_t* lut = geob ? (dc_lut ? lut_dc + dctx * LUT_BUCKETS : lut_run) : lut_lvl + lc * LUT_BUCKETS;
        const uint16_t* cum = geob ? cum_dc + dctx * CUM_LEN : cum_lvl + lc * CUM_LEN;
        const bool use_lut = !geob || dc_lut;
        const uint32_t sc = dl_sym<true>(L, lut, use_lut, cum);
        m = dl_suffix(L, sc);
        if (!geob) {
            err |= m > mlv ? 1u : 0u;
            blk[idx] = (int32_t)m;
            pcat = sc;
            has = true;
            pos = idx + 1u;
            lc0 = ctl[by_pos ? pos : sc];
        } else {
            ++b;
            blk += 64;
            bx = bx + 1u == cols ? 0u : bx + 1u;
            const bool ht = b >= cols;
            err |= m > mdc ? 1u : 0u;
            dcv = (int64_t)dc_pred(bx != 0u, left, ht, top_next) + unmap_s(m);
            err |= (dcv > dlim || dcv < -dlim) ? 1u : 0u;
            left = (int32_t)dcv;
            blk[0] = left;
            top_next = (b + 1u < nblk && b + 1u >= cols) ? blk[64 - (int64_t)cols * 64] : 0;
            prev_dcc = sc;
            pos = 1u;
            pcat = 0u;
            has = false;
            lc0 = ctl[by_pos ? 1u : 79u];
        }
    }
#undef DCH_FINISH
    if (err == 0u && dl_consumed(L) != nbytes) { err = 1u; }
    status[si] = err != 0u ? TCG_ERR_MALFORMED : 0;
}

// ------------------------------------------------------------------ reconstruction
//
// Blocks are reconstructed 32 to a CTA of 256 threads (RB_BLOCKS). Lane b of
// warp 0 first gathers block b's facts (quantiser steps, clamp, destination).
// Then every thread loads two 16-byte pieces of the CTA's 8 KB of
// coefficients (contiguous, so each warp reads 512 bytes in one go) and
// dequantises them into natural order in shared memory; warp w runs the
// 8-point row pass of row w of all 32 blocks (lane = block), then the column
// pass of column w, and finally stores row w of every block, 16 bytes per
// lane, so a warp writes 512 contiguous bytes of a plane row when the blocks
// lie side by side. The arithmetic is idct8x8's, split at its passes:
// G = c (.) W, B = G * M, xhat = round(M^T * B / 2^32).
constexpr uint32_t RB_BLOCKS = 32u;
constexpr uint32_t RB_CP = 65u;   // words per block in the coefficient and B arrays (odd: no bank conflicts)
constexpr uint32_t RB_TP = 72u;   // samples per block in the output tile (144 B rows of 16-byte pieces)

struct RBlock {
    const uint32_t* Q;  // quantiser steps, natural order
    uint16_t* dst;      // the block's top-left visible sample
    int64_t fc;         // dequantised coefficient clamp
    uint32_t pitch;     // plane row pitch in samples
    uint32_t cw, ch;    // visible columns and rows of the block
    uint32_t climit;    // highest zigzag position kept
    uint32_t bd;
    uint32_t ok;        // 0: nothing to write (past the batch, concealed slice, outside the plane)
    uint32_t vec;       // whole rows of 16-byte aligned samples
};

struct RShared {
    int32_t c[RB_BLOCKS * RB_CP];
    int64_t B[RB_BLOCKS * RB_CP];
    __align__(16) uint16_t t[RB_BLOCKS * RB_TP];
    RBlock blk[RB_BLOCKS];
    uint8_t zz[64];
};

// The transform tables as doubles (exact) for the double-precision passes.
__device__ __constant__ double c_tmd[64] = {
    13, 13, 13, 13, 13, 13, 13, 13, 13, 11, 7, 1, -1, -7, -11, -13,
    12, 5, -5, -12, -12, -5, 5, 12, 11, -4, -13, -8, 8, 13, 4, -11,
    9, -9, -9, 9, 9, -9, -9, 9, 8, -13, 4, 11, -11, -4, 13, -8,
    5, -12, 12, -5, -5, 12, -12, 5, 1, -7, 11, -13, 13, -11, 7, -1};
__device__ __constant__ double c_twd[64] = {
    2350, 4672, 4699, 4293, 4902, 4293, 4699, 4672,
    4672, 9288, 9343, 8535, 9747, 8535, 9343, 9288,
    4699, 9343, 9399, 8586, 9805, 8586, 9399, 9343,
    4293, 8535, 8586, 7843, 8957, 7843, 8586, 8535,
    4902, 9747, 9805, 8957, 10228, 8957, 9805, 9747,
    4293, 8535, 8586, 7843, 8957, 7843, 8586, 8535,
    4699, 9343, 9399, 8586, 9805, 8586, 9399, 9343,
    4672, 9288, 9343, 8535, 9747, 8535, 9343, 9288};

// round_shift32 of an integer-valued double below 2^53 in magnitude: |v| + 2^31
// and its scaling by 2^-32 are exact, so the floor is the integer form's
// sign-split rounding
__device__ __forceinline__ int32_t round_shift32_f64(double v)
{
    const double r = floor((fabs(v) + 2147483648.0) * 2.3283064365386962890625e-10);
    return v >= 0.0 ? (int32_t)r : -(int32_t)r;
}

__device__ __forceinline__ int64_t recon_clamp(uint32_t bd)
{
    return bd <= 12u ? ((int64_t)1 << 25) : (((int64_t)1 << 25) * (int64_t)((1u << (bd - 1u)) - 1u)) / 2047;
}

// Phases 1-4 above; sh.blk is filled and visible (after a barrier) on entry.
// coef points at block gb0 and holds nvalid blocks from there.
// The CTA's coefficients, loaded before the block facts are gathered so that
// the loads overlap the lookups.
__device__ __forceinline__ void recon_preload(const int32_t* __restrict__ coef, uint32_t nvalid, int4 pre[2])
{
#pragma unroll
    for (uint32_t h = 0; h < 2u; ++h) {
        const uint32_t idx = threadIdx.x + 256u * h;
        pre[h] = (idx >> 4) < nvalid ? __ldg(reinterpret_cast<const int4*>(coef) + idx) : make_int4(0, 0, 0, 0);
    }
}

__device__ __forceinline__ void recon_blocks(RShared& sh, const int4 pre[2], uint32_t nvalid)
{
    const uint32_t t = threadIdx.x, w = t >> 5, lane = t & 31u;
    // dequantise into natural order
#pragma unroll
    for (uint32_t h = 0; h < 2u; ++h) {
        const uint32_t idx = t + 256u * h;  // 16-byte piece of the CTA's coefficients
        const uint32_t b = idx >> 4, i0 = (idx & 15u) * 4u;
        const RBlock& R = sh.blk[b];
        if (b < nvalid && R.ok) {
            const int4 v = pre[h];
            const int32_t vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (uint32_t j = 0; j < 4u; ++j) {
                const uint32_t i = i0 + j;
                int32_t lv = i == 0u ? vv[j] : unmap_s((uint32_t)vv[j]);
                lv = i <= R.climit ? lv : 0;
                const uint32_t nat = sh.zz[i];
                int64_t f = (int64_t)lv * __ldg(R.Q + nat);
                f = f > R.fc ? R.fc : (f < -R.fc ? -R.fc : f);
                sh.c[b * RB_CP + nat] = (int32_t)f;
            }
        }
    }
    __syncthreads();
    const uint32_t b = lane;
    const bool live = b < nvalid && sh.blk[b].ok;
    // Up to 12 bits the dequantised coefficients are within +-2^25, so every
    // product and partial sum of both passes is an integer below 2^51 in
    // magnitude (|W| < 2^14, column sums of |M| are at most 72) and double
    // arithmetic gives the 64-bit integer results exactly, one fused
    // multiply-add per term; wider samples take the 64-bit integer passes.
    const bool f64 = live && sh.blk[b].bd <= 12u;
    if (live) {  // row pass: row u = w
        const uint32_t u = w;
        if (f64) {
            double g[8];
#pragma unroll
            for (int v = 0; v < 8; ++v) { g[v] = (double)sh.c[b * RB_CP + u * 8u + v] * c_twd[u * 8u + v]; }
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                double pe = g[0] * c_tmd[x], po = g[1] * c_tmd[8 + x];
#pragma unroll
                for (int v = 2; v < 8; v += 2) { pe = fma(g[v], c_tmd[v * 8 + x], pe); po = fma(g[v + 1], c_tmd[(v + 1) * 8 + x], po); }
                sh.B[b * RB_CP + u * 8u + x] = __double_as_longlong(pe + po);
                sh.B[b * RB_CP + u * 8u + 7u - x] = __double_as_longlong(pe - po);
            }
        } else {
            int64_t g[8];
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                int32_t c = sh.c[b * RB_CP + u * 8u + v];
                c = c > (1 << 30) ? (1 << 30) : (c < -(1 << 30) ? -(1 << 30) : c);
                g[v] = (int64_t)c * c_tw[u * 8u + v];
            }
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                int64_t pe = 0, po = 0;
#pragma unroll
                for (int v = 0; v < 8; v += 2) { pe += g[v] * TCG_M(v, x); po += g[v + 1] * TCG_M(v + 1, x); }
                sh.B[b * RB_CP + u * 8u + x] = pe + po;
                sh.B[b * RB_CP + u * 8u + 7u - x] = pe - po;
            }
        }
    }
    __syncthreads();
    if (live) {  // column pass: column x = w
        const uint32_t x = w;
        const int32_t mid = 1 << (sh.blk[b].bd - 1u), maxv = (1 << sh.blk[b].bd) - 1;
        int32_t out[8];
        if (f64) {
            double Bc[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) { Bc[u] = __longlong_as_double(sh.B[b * RB_CP + u * 8u + x]); }
#pragma unroll
            for (int y = 0; y < 4; ++y) {
                double qe = c_tmd[y] * Bc[0], qo = c_tmd[8 + y] * Bc[1];
#pragma unroll
                for (int u = 2; u < 8; u += 2) { qe = fma(c_tmd[u * 8 + y], Bc[u], qe); qo = fma(c_tmd[(u + 1) * 8 + y], Bc[u + 1], qo); }
                out[y] = round_shift32_f64(qe + qo);
                out[7 - y] = round_shift32_f64(qe - qo);
            }
        } else {
            int64_t Bc[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) { Bc[u] = sh.B[b * RB_CP + u * 8u + x]; }
#pragma unroll
            for (int y = 0; y < 4; ++y) {
                int64_t qe = 0, qo = 0;
#pragma unroll
                for (int u = 0; u < 8; u += 2) { qe += (int64_t)TCG_M(u, y) * Bc[u]; qo += (int64_t)TCG_M(u + 1, y) * Bc[u + 1]; }
                out[y] = round_shift32(qe + qo);
                out[7 - y] = round_shift32(qe - qo);
            }
        }
#pragma unroll
        for (int y = 0; y < 8; ++y) {
            const int32_t a = out[y] + mid;
            sh.t[b * RB_TP + y * 8u + x] = (uint16_t)(a < 0 ? 0 : (a > maxv ? maxv : a));
        }
    }
    __syncthreads();
    if (live) {  // store row y = w
        const RBlock& R = sh.blk[b];
        const uint32_t y = w;
        if (y < R.ch) {
            uint16_t* d = R.dst + (size_t)y * R.pitch;
            const uint16_t* s = sh.t + b * RB_TP + y * 8u;
            if (R.vec) {
                *reinterpret_cast<uint4*>(d) = *reinterpret_cast<const uint4*>(s);
            } else {
                for (uint32_t x = 0; x < R.cw; ++x) { d[x] = s[x]; }
            }
        }
    }
}

// ------------------------------------------------------------------ V8 segments
//
// V8 (reference codec.c:4321-4475 segment decode, 4772-4975 frame decode).
// Tile tables hold every row at a fixed place (flags, DC rows 0..4, run row,
// level rows 0..4: 350 bytes), so k_v8_dtab builds the same decode-table
// layout as k_dtables from them. A warp decodes up to 32 segments of one
// tile, one lane each, with the tile's eleven bucket tables and cumulative
// tables in shared memory (12.5 KB). DC prediction and the DC context stay
// inside the segment (left = the segment's previous block in raster order,
// top = the block one plane row up when the segment reaches back that far).
// Magnitude and DC-domain checks use the 12-bit limits at every bit depth,
// as the reference's segment decoder does. A segment that fails is zeroed,
// so it reconstructs at the mid level, the reference's concealment.

constexpr uint32_t V8_TABLE_BYTES = 350u;
constexpr uint32_t V8D_LUT = 0u;                                  // 11 x 1 KB bucket tables
constexpr uint32_t V8D_CUM = MAX_CTX * LUT_BYTES;                 // 11 x 66 u16
constexpr uint32_t V8D_SMEM = V8D_CUM + DCH_CUM_BYTES;
// per plane of a batch: first block, first segment, block columns, visible
// width and height, output offset / 64, segment blocks log2, bit depth
constexpr uint32_t V8_PINFO = 8u;

// one block per tile: CRC of the table and the member streams against the stored one
__global__ void __launch_bounds__(256) k_v8_tcrc(const tcg_v8_tile* __restrict__ tiles, const uint8_t* __restrict__ pkt,
                                                 const uint32_t* __restrict__ crctab, uint8_t* __restrict__ ok)
{
    __shared__ uint32_t t[8 * 256];
    __shared__ uint32_t scratch[512];
    __shared__ uint32_t c_tab;
    for (uint32_t i = threadIdx.x; i < 8u * 256u; i += blockDim.x) { t[i] = crctab[i]; }
    __syncthreads();
    const tcg_v8_tile& T = tiles[blockIdx.x];
    const uint32_t c1 = crc32_block(pkt + T.table_off, V8_TABLE_BYTES, t, scratch);
    if (threadIdx.x == 0) { c_tab = c1; }
    __syncthreads();
    const uint32_t c2 = crc32_block(pkt + T.stream_off, T.stream_bytes, t, scratch);
    if (threadIdx.x == 0) {
        const uint32_t c = T.stream_bytes == 0u ? c_tab : crc_combine(c_tab, c2, gf2_xpow8n(T.stream_bytes));
        ok[blockIdx.x] = c == T.crc ? 1u : 0u;
    }
}

// one warp per tile: decode tables in k_dtables' layout from the fixed rows
// (the host has checked the flags and that every used row normalises)
__global__ void __launch_bounds__(32) k_v8_dtab(const tcg_v8_tile* __restrict__ tiles, const uint8_t* __restrict__ pkt,
                                                uint8_t* __restrict__ tabs)
{
    const tcg_v8_tile& T = tiles[blockIdx.x];
    const uint8_t* tb350 = pkt + T.table_off;
    uint8_t* tb = tabs + (size_t)blockIdx.x * DTAB_BYTES;
    const uint32_t t = threadIdx.x;
    const uint32_t fl = tb350[0], lm = fl & 3u, dm = (fl >> 2) & 1u;
    const uint32_t nd = dm ? DCP_CTX : 1u, nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u;
    const uint32_t nrows = nd + 1u + nl;
    if (t < nrows) {
        uint32_t ctx, off, n;
        if (t < nd) { ctx = t; off = 1u + t * DC_SYMS; n = DC_SYMS; }
        else if (t == nd) { ctx = 5u; off = 1u + DCP_CTX * DC_SYMS; n = RUN_SYMS; }
        else { ctx = 6u + (t - nd - 1u); off = 1u + DCP_CTX * DC_SYMS + RUN_SYMS + (t - nd - 1u) * LVL_SYMS; n = LVL_SYMS; }
        uint8_t bytes[64];
        for (uint32_t k = 0; k < n; ++k) { bytes[k] = tb350[off + k]; }
        uint16_t fr[64], cu[64];
        if (model_from_bytes(bytes, n, fr, cu)) {
            uint16_t* cd = reinterpret_cast<uint16_t*>(tb + TAB_CUM + (size_t)ctx * CUM_BYTES);
            for (uint32_t k = 0; k < CUM_LEN; ++k) { cd[k] = k < n ? cu[k] : (uint16_t)4096u; }
            uint32_t* lut = reinterpret_cast<uint32_t*>(tb + TAB_LUT + (size_t)ctx * LUT_BYTES);
            for (uint32_t sy = 0; sy < n; ++sy) {
                const uint32_t c0 = cu[sy], c1 = c0 + fr[sy];
                for (uint32_t bk = (c0 + 15u) >> 4; bk < LUT_BUCKETS && (bk << 4) < c1; ++bk) { lut[bk] = c0 | (sy << 12); }
            }
        }
    }
    if (t == 0) {
        uint32_t* hdr = reinterpret_cast<uint32_t*>(tb + TAB_HDR);
        hdr[0] = lm; hdr[1] = dm; hdr[2] = 0u;
    }
}

// One thread per segment, up to V8DC_LANES segments of one tile per CTA: the
// tile's tables are staged once per CTA, so four warps share 12.5 KB of shared
// memory (one warp per CTA left the SMs at about 14 resident warps, too few to
// hide the chains' latency).
constexpr uint32_t V8DC_LANES = 128u;

__global__ void __launch_bounds__(V8DC_LANES) k_v8_dchain(const tcg_v8_seg* __restrict__ segs, const uint32_t* __restrict__ wtile,
                                                  const int32_t* __restrict__ wsegs, const uint32_t* __restrict__ pinfo,
                                                  const uint8_t* __restrict__ tile_ok, const uint8_t* __restrict__ pkt,
                                                  const uint8_t* __restrict__ tabs, int32_t* __restrict__ coef,
                                                  uint8_t* __restrict__ seg_fail)
{
    extern __shared__ __align__(16) uint8_t vsm[];
    const uint32_t lane = threadIdx.x;
    const uint32_t ti = wtile[blockIdx.x];
    if (tile_ok[ti] == 0u) { return; }  // concealed whole: coefficients stay zero
    const uint8_t* tb = tabs + (size_t)ti * DTAB_BYTES;
    for (uint32_t k = lane; k < V8D_SMEM / 16u; k += V8DC_LANES) {
        reinterpret_cast<uint4*>(vsm)[k] = reinterpret_cast<const uint4*>(tb)[k];
    }
    __syncthreads();
    const int32_t si = wsegs[blockIdx.x * V8DC_LANES + lane];
    if (si < 0) { return; }
    const tcg_v8_seg& S = segs[si];
    const uint32_t* hdr = reinterpret_cast<const uint32_t*>(tb + TAB_HDR);
    const uint32_t lm = hdr[0], dm = hdr[1];
    const uint32_t* luts = reinterpret_cast<const uint32_t*>(vsm + V8D_LUT);
    const uint16_t* cums = reinterpret_cast<const uint16_t*>(vsm + V8D_CUM);
    const uint32_t cols = pinfo[V8_PINFO * S.plane + 2u];
    int32_t* blk = coef + ((size_t)pinfo[V8_PINFO * S.plane] + S.blk0) * 64u;
    DLane L;
    dl_init(L, pkt + S.off, S.len);
    uint32_t err = L.x < RANS_L ? 1u : 0u;
    uint32_t prev_dcc = 0u;
    int32_t left = 0;
    for (uint32_t i = 0; i < S.nblk && err == 0u; ++i) {
        const uint32_t dctx = (i == 0u || dm == 0u) ? 0u : dcp_ctx(prev_dcc, true);
        const uint32_t dcat = dl_sym<true>(L, luts + dctx * LUT_BUCKETS, true, cums + dctx * CUM_LEN);
        uint32_t m = dl_suffix(L, dcat);
        err |= m > 0x08000000u ? 1u : 0u;
        const int32_t top = i >= cols ? blk[(size_t)(i - cols) * 64u] : 0;
        const int64_t dcv = (int64_t)dc_pred(i != 0u, left, i >= cols, top) + unmap_s(m);
        err |= (dcv > ((int64_t)1 << 25) || dcv < -((int64_t)1 << 25)) ? 1u : 0u;
        int32_t* b = blk + (size_t)i * 64u;
        b[0] = (int32_t)dcv;
        left = (int32_t)dcv;
        prev_dcc = dcat;
        uint32_t pos = 1u, pcat = 0u;
        bool has = false;
        while (err == 0u) {
            const uint32_t r = dl_sym<false>(L, luts + 5u * LUT_BUCKETS, true, cums + 5u * CUM_LEN);
            if (r == 63u) { break; }
            const uint32_t idx = pos + r;
            if (idx > 63u) { err = 1u; break; }
            const uint32_t lc = 6u + (lm == 1u ? pos_ctx(idx) : (lm == 2u ? prev_ctx(pcat, has) : 0u));
            const uint32_t cat = dl_sym<true>(L, luts + lc * LUT_BUCKETS, true, cums + lc * CUM_LEN);
            m = dl_suffix(L, cat);
            err |= m > 0x04000000u ? 1u : 0u;
            b[idx] = (int32_t)m;  // zigzag-mapped level at zigzag position idx
            pcat = cat;
            has = true;
            pos = idx + 1u;
        }
    }
    if (err == 0u && dl_consumed(L) != S.len) { err = 1u; }
    if (err != 0u) {
        for (uint32_t k = 0; k < S.nblk * 64u; ++k) { blk[k] = 0; }
    }
    seg_fail[si] = err != 0u ? 1u : 0u;
}

// Reconstruction of every block of the batch's planes (k_didct's
// arithmetic): the block's plane from the unit map, its segment by the
// plane's segment size, its quantiser steps by the segment.
__global__ void __launch_bounds__(256) k_v8_didct(const tcg_v8_seg* __restrict__ segs, const uint32_t* __restrict__ pinfo,
                                                  uint32_t nplanes, const uint32_t* __restrict__ q,
                                                  const int32_t* __restrict__ coef, uint32_t total,
                                                  const uint32_t* __restrict__ umap, uint16_t* __restrict__ out)
{
    __shared__ RShared sh;
    const uint32_t gb0 = blockIdx.x * RB_BLOCKS;
    const uint32_t nvalid = min(RB_BLOCKS, total - gb0);
    int4 pre[2];
    recon_preload(coef + (size_t)gb0 * 64u, nvalid, pre);
    if (threadIdx.x < 64u) { sh.zz[threadIdx.x] = k_zigzag[threadIdx.x]; }
    if (threadIdx.x < RB_BLOCKS) {
        RBlock R;
        R.ok = 0u;
        const uint32_t gb = gb0 + threadIdx.x;
        if (gb < total) {
            const uint32_t* I = pinfo + V8_PINFO * unit_of(pinfo, V8_PINFO, nplanes, umap[blockIdx.x], gb);
            const uint32_t lb = gb - I[0];
            const uint32_t cols = I[2], vis_w = I[3], vis_h = I[4], sb_log2 = I[6], bd = I[7];
            const tcg_v8_seg& S = segs[I[1] + (lb >> sb_log2)];
            const uint32_t px = (lb % cols) * 8u, py = (lb / cols) * 8u;
            if (px < vis_w && py < vis_h) {
                R.ok = 1u;
                R.Q = q + (size_t)S.qidx * 64u;
                R.dst = out + (size_t)I[5] * 64u + (size_t)py * vis_w + px;
                R.fc = recon_clamp(bd);
                R.pitch = vis_w;
                R.cw = min(8u, vis_w - px);
                R.ch = min(8u, vis_h - py);
                R.climit = 63u;
                R.bd = bd;
                R.vec = R.cw == 8u && (vis_w & 7u) == 0u;
            }
        }
        sh.blk[threadIdx.x] = R;
    }
    __syncthreads();
    recon_blocks(sh, pre, nvalid);
}

// ------------------------------------------------------------------ chain, warp tiling
//
// Second tiling of the same decode (the tuner below picks per batch size):
// one warp decodes one slice. The coder state is warp-uniform; lane j holds the
// frequency and cumulative start of symbol j (and j+32 for the 64-symbol run
// alphabet) of every context the slice uses, so a symbol search is one compare
// per lane and the matching lane's next state is broadcast with a warp OR
// reduction (exactly one lane matches: the alphabet partitions 0..4095).
// Stream bytes come through a 64-bit bit window refilled one word at a time
// from 128-byte chunks that the lanes load one chunk ahead. Error conditions
// accumulate in a flag and end the slice at the next block boundary: any
// error conceals the slice, so only whether one occurred matters, and reading
// past the payload is harmless because it can only add to a consumed-byte
// count that must end equal to the payload size.

#define FULL_MASK 0xFFFFFFFFu

struct Win {
    uint32_t x;            // coder state
    uint32_t whi, wlo;     // upcoming stream bits, first bit in the MSB of whi
    uint32_t wbits;        // valid bits in whi:wlo
    uint32_t cb;           // stream bytes moved into the state
    uint32_t cur, nxt;     // lane j: word j of the current / next 128-byte chunk (big-endian)
    uint32_t k;            // next word of the current chunk
    const uint32_t* cp;    // aligned start of the chunk after the next one
    const uint32_t* lim;   // one past the last word that overlaps the payload
};

__device__ __forceinline__ uint32_t win_load(const uint32_t* p, const uint32_t* lim)
{
    return p < lim ? __byte_perm(__ldg(p), 0u, 0x0123u) : 0u;
}

__device__ __forceinline__ uint32_t win_take(Win& w, uint32_t lane)
{
    const uint32_t word = __shfl_sync(FULL_MASK, w.cur, w.k);
    w.k += 1u;
    if (w.k == 32u) {
        w.k = 0u;
        w.cur = w.nxt;
        w.nxt = win_load(w.cp + lane, w.lim);
        w.cp += 32;
    }
    return word;
}

// keep at least 32 bits in the window (called after every renormalisation,
// which consumes at most 24)
__device__ __forceinline__ void win_refill(Win& w, uint32_t lane)
{
    if (w.wbits < 32u) {
        const uint32_t word = win_take(w, lane);
        w.whi |= word >> w.wbits;
        w.wlo |= word << (32u - w.wbits);
        w.wbits += 32u;
    }
}

// state <- xn followed by as many stream bytes as bring it to [2^23, ...)
__device__ __forceinline__ void win_renorm(Win& w, uint32_t xn, uint32_t lane)
{
    const bool c1 = xn < RANS_L, c2 = xn < (RANS_L >> 8), c3 = xn < (RANS_L >> 16);
    const uint32_t x8 = __funnelshift_l(w.whi, xn, 8);
    const uint32_t x16 = __funnelshift_l(w.whi, xn, 16);
    const uint32_t x24 = __funnelshift_l(w.whi, xn, 24);
    w.x = c2 ? (c3 ? x24 : x16) : (c1 ? x8 : xn);
    const uint32_t n8 = c2 ? (c3 ? 24u : 16u) : (c1 ? 8u : 0u);
    w.whi = __funnelshift_l(w.wlo, w.whi, n8);
    w.wlo <<= n8;
    w.wbits -= n8;
    w.cb += n8 >> 3;
    win_refill(w, lane);
}

__device__ __forceinline__ void win_init(Win& w, const uint8_t* b, uint32_t n, uint32_t lane)
{
    const uintptr_t a = (uintptr_t)b;
    const uint32_t* base = reinterpret_cast<const uint32_t*>(a & ~(uintptr_t)127);
    w.lim = reinterpret_cast<const uint32_t*>((a + n + 3u) & ~(uintptr_t)3);
    w.cur = win_load(base + lane, w.lim);
    w.nxt = win_load(base + 32 + lane, w.lim);
    w.cp = base + 64;
    const uint32_t off = (uint32_t)(a & 127u);
    w.k = off >> 2;
    const uint32_t a8 = (off & 3u) * 8u;
    const uint32_t w0 = win_take(w, lane);
    const uint32_t w1 = win_take(w, lane);
    w.x = __funnelshift_l(w1, w0, a8);  // first four payload bytes, big-endian
    w.whi = w1 << a8;
    w.wlo = 0u;
    w.wbits = 32u - a8;
    w.cb = 4u;
    win_refill(w, lane);
}

// one symbol of an alphabet of at most 32 (lane j holds symbol j)
__device__ __forceinline__ uint32_t dec_sym32(Win& w, uint32_t f, uint32_t c, uint32_t lane)
{
    const uint32_t x = w.x;
    const uint32_t d = (x & 4095u) - c;
    const bool in = d < f;
    const uint32_t xn = f * (x >> 12) + d;
    const uint32_t xv = __reduce_or_sync(FULL_MASK, in ? xn : 0u);
    const uint32_t s = __reduce_or_sync(FULL_MASK, in ? lane : 0u);
    win_renorm(w, xv, lane);
    return s;
}

// one symbol of a 64-symbol alphabet (lane j holds symbols j and j+32)
__device__ __forceinline__ uint32_t dec_sym64(Win& w, uint32_t fa, uint32_t ca, uint32_t fb, uint32_t cb,
                                              uint32_t lane)
{
    const uint32_t x = w.x;
    const uint32_t slot = x & 4095u, xs = x >> 12;
    const uint32_t da = slot - ca, db = slot - cb;
    const bool ia = da < fa, ib = db < fb;
    const uint32_t v = ia ? fa * xs + da : (ib ? fb * xs + db : 0u);
    const uint32_t xv = __reduce_or_sync(FULL_MASK, v);
    const uint32_t s = __reduce_or_sync(FULL_MASK, ia ? lane : (ib ? lane + 32u : 0u));
    win_renorm(w, xv, lane);
    return s;
}

// raw chunk of wd bits (wd <= 23)
__device__ __forceinline__ uint32_t dec_chunk(Win& w, uint32_t wd, uint32_t lane)
{
    const uint32_t v = w.x & ~(0xFFFFFFFFu << wd);
    win_renorm(w, w.x >> wd, lane);
    return v;
}

// category suffix: m = 2^(cat-1) | (cat-1 raw bits), split 16 + rest above 23
__device__ __forceinline__ uint32_t dec_suffix(Win& w, uint32_t cat, uint32_t lane)
{
    const uint32_t b = cat > 1u ? cat - 1u : 0u;
    uint32_t v;
    if (b <= 23u) {
        v = dec_chunk(w, b, lane);
    } else {
        const uint32_t lo = dec_chunk(w, 16u, lane);
        v = (dec_chunk(w, b - 16u, lane) << 16) | lo;
    }
    return cat == 0u ? 0u : (1u << (cat - 1u)) | v;
}

template <uint32_t LM, uint32_t DM>
__device__ __forceinline__ int32_t dchain_slice(const DSlice& S, const DPlane& P, const uint8_t* __restrict__ tb,
                                                const uint8_t* __restrict__ stream, uint32_t nbytes,
                                                int32_t* __restrict__ coef, int32_t* __restrict__ rows)
{
    const uint32_t lane = threadIdx.x & 31u;
    // per-lane model entries
    constexpr uint32_t ND = DM ? 5u : 1u;
    constexpr uint32_t NL = LM == 1u ? 4u : (LM == 2u ? 5u : 1u);
    uint32_t dcf[ND], dcc[ND], lvf[NL], lvc[NL];
    auto ent = [&](uint32_t ctx, uint32_t s, uint32_t& f, uint32_t& c) {
        const uint16_t* cu = reinterpret_cast<const uint16_t*>(tb + TAB_CUM + (size_t)ctx * CUM_BYTES);
        c = cu[s];
        f = (uint32_t)cu[s + 1u] - cu[s];  // 0 past the alphabet and for unused symbols
    };
#pragma unroll
    for (uint32_t i = 0; i < ND; ++i) { ent(i, lane, dcf[i], dcc[i]); }
#pragma unroll
    for (uint32_t i = 0; i < NL; ++i) { ent(6u + i, lane, lvf[i], lvc[i]); }
    uint32_t rfa, rca, rfb, rcb;
    ent(5u, lane, rfa, rca);
    ent(5u, lane + 32u, rfb, rcb);

    Win w;
    win_init(w, stream, nbytes, lane);
    uint32_t err = w.x < RANS_L ? 1u : 0u;
    const bool wide = P.bd > 12u;
    const uint32_t mdc = wide ? 0x0FFFFFFFu : 0x08000000u;
    const uint32_t mlv = wide ? 0x07FFFFFFu : 0x04000000u;
    const int64_t dlim = wide ? ((int64_t)1 << 27) : ((int64_t)1 << 25);
    int32_t* prow = rows;
    int32_t* crow = rows + S.cols;
    uint32_t prev_dcc = 0;
    bool first = true;
    for (uint32_t by = 0; by < S.bh && err == 0u; ++by) {
        int32_t left = 0;
        for (uint32_t bx = 0; bx < S.cols; ++bx) {
            // DC
            uint32_t f0 = dcf[0], c0 = dcc[0];
            if (DM) {
                const uint32_t dctx = first ? 0u : dcp_ctx(prev_dcc, true);
#pragma unroll
                for (uint32_t i = 1; i < ND; ++i) {
                    f0 = dctx == i ? dcf[i] : f0;
                    c0 = dctx == i ? dcc[i] : c0;
                }
            }
            const int32_t top = by != 0u ? prow[bx] : 0;
            const uint32_t dcat = dec_sym32(w, f0, c0, lane);
            const uint32_t dmv = dec_suffix(w, dcat, lane);
            err |= dmv > mdc ? 1u : 0u;
            const int32_t pred = dc_pred(bx != 0u, left, by != 0u, top);
            const int64_t dcv = (int64_t)pred + unmap_s(dmv);
            err |= (dcv > dlim || dcv < -dlim) ? 1u : 0u;
            left = (int32_t)dcv;
            if (lane == 0u) { crow[bx] = left; }
            prev_dcc = dcat;
            first = false;
            int32_t clo = lane == 0u ? left : 0, chi = 0;
            // AC: (run, level, suffix) until the end-of-block run symbol
            uint32_t pos = 1u, pcat = 0u;
            bool has = false;
            for (;;) {
                const uint32_t r = dec_sym64(w, rfa, rca, rfb, rcb, lane);
                const uint32_t idx = pos + r;
                if (r == 63u || idx > 63u) {
                    err |= r != 63u ? 1u : 0u;
                    break;
                }
                uint32_t fl = lvf[0], cl = lvc[0];
                if (LM != 0u) {
                    const uint32_t lc = LM == 1u ? pos_ctx(idx) : prev_ctx(pcat, has);
#pragma unroll
                    for (uint32_t i = 1; i < NL; ++i) {
                        fl = lc == i ? lvf[i] : fl;
                        cl = lc == i ? lvc[i] : cl;
                    }
                }
                const uint32_t cat = dec_sym32(w, fl, cl, lane);
                const uint32_t m = dec_suffix(w, cat, lane);
                err |= m > mlv ? 1u : 0u;
                const int32_t v = (int32_t)m;  // zigzag-mapped level at zigzag position idx
                if ((idx & 31u) == lane) {
                    if (idx & 32u) { chi = v; } else { clo = v; }
                }
                pcat = cat;
                has = true;
                pos = idx + 1u;
            }
            int32_t* blk = coef + (size_t)(S.blk0 + by * S.cols + bx) * 64u;
            blk[lane] = clo;
            blk[32u + lane] = chi;
            if (err != 0u) { break; }
        }
        __syncwarp();
        int32_t* sw = prow; prow = crow; crow = sw;
    }
    if (err == 0u && w.cb != nbytes) { err = 1u; }
    return err != 0u ? TCG_ERR_MALFORMED : 0;
}

// One warp per colour slice (one warp per block, so every slice of a batch is
// resident at once); dynamic shared memory holds two DC rows of the slice.
__global__ void __launch_bounds__(32) k_dchain_w(const DSlice* __restrict__ slices, const uint32_t* __restrict__ cslices,
                                               const DPlane* __restrict__ planes, const uint8_t* __restrict__ pkt,
                                               const uint8_t* __restrict__ tabs, int32_t* __restrict__ coef,
                                               int32_t* __restrict__ status)
{
    extern __shared__ __align__(16) int32_t rows[];
    const uint32_t si = cslices[blockIdx.x];
    if (status[si] != 0) { return; }
    const DSlice& S = slices[si];
    const DPlane& P = planes[S.plane];
    const uint8_t* tb = tabs + (size_t)blockIdx.x * DTAB_BYTES;
    const uint32_t* hdr = reinterpret_cast<const uint32_t*>(tb + TAB_HDR);
    const uint32_t lm = hdr[0], dm = hdr[1], plen = hdr[2];
    const uint8_t* stream = pkt + S.pay + plen;
    const uint32_t nb = S.size - plen;
    int32_t rc;
    switch (lm * 2u + dm) {
    case 0: rc = dchain_slice<0, 0>(S, P, tb, stream, nb, coef, rows); break;
    case 1: rc = dchain_slice<0, 1>(S, P, tb, stream, nb, coef, rows); break;
    case 2: rc = dchain_slice<1, 0>(S, P, tb, stream, nb, coef, rows); break;
    case 3: rc = dchain_slice<1, 1>(S, P, tb, stream, nb, coef, rows); break;
    case 4: rc = dchain_slice<2, 0>(S, P, tb, stream, nb, coef, rows); break;
    default: rc = dchain_slice<2, 1>(S, P, tb, stream, nb, coef, rows); break;
    }
    if (threadIdx.x == 0) { status[si] = rc; }
}

// ------------------------------------------------------------------ reconstruction
//
// Coefficient blocks are in zigzag order, as the chains decode them: the DC
// value at index 0 (signed) and the AC levels in their zigzag-mapped form
// (m = 2v or -2v-1); 0 maps to 0, so untouched positions read as zero levels.
// Reconstruction places them in natural order while loading.

// The block's colour slice is found by a binary search over the colour slices,
// which are in increasing order of their first block.
__global__ void __launch_bounds__(256) k_didct(const DSlice* __restrict__ slices, const uint32_t* __restrict__ cslices,
                                               uint32_t ncs,
                                               const uint32_t* __restrict__ slice_tab, const DPlane* __restrict__ planes,
                                               const uint8_t* __restrict__ tabs, const int32_t* __restrict__ coef,
                                               const int32_t* __restrict__ status, uint32_t total,
                                               const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ umap,
                                               uint16_t* __restrict__ out)
{
    __shared__ RShared sh;
    const uint32_t gb0 = blockIdx.x * RB_BLOCKS;
    const uint32_t nvalid = min(RB_BLOCKS, total - gb0);
    int4 pre[2];
    recon_preload(coef + (size_t)gb0 * 64u, nvalid, pre);
    if (threadIdx.x < 64u) { sh.zz[threadIdx.x] = k_zigzag[threadIdx.x]; }
    if (threadIdx.x < RB_BLOCKS) {
        RBlock R;
        R.ok = 0u;
        const uint32_t gb = gb0 + threadIdx.x;
        if (gb < total) {
            const uint32_t si = cslices[unit_of(cstart, 1u, ncs, umap[blockIdx.x], gb)];
            if (status[si] == 0) {
                const DSlice& S = slices[si];
                const DPlane& P = planes[S.plane];
                const uint32_t lb = gb - S.blk0;
                const uint32_t px = (lb % S.cols) * 8u, py = (S.y0 + lb / S.cols) * 8u;
                R.ok = 1u;
                R.Q = reinterpret_cast<const uint32_t*>(tabs + (size_t)slice_tab[si] * DTAB_BYTES + TAB_Q);
                R.dst = out + P.out_off + (size_t)py * P.vis_w + px;
                R.fc = recon_clamp(P.bd);
                R.pitch = P.vis_w;
                R.cw = min(8u, P.vis_w - px);
                R.ch = min(8u, P.vis_h - py);
                R.climit = P.climit;  // reduced delivery drops the high zigzag positions
                R.bd = P.bd;
                R.vec = R.cw == 8u && (P.vis_w & 7u) == 0u;
            }
        }
        sh.blk[threadIdx.x] = R;
    }
    __syncthreads();
    recon_blocks(sh, pre, nvalid);
}

// Scaled delivery (reference color_store.h:223-313 scaled samples,
// codec.c:7955-7964 alpha, 7987-8000 concealment): target sample (x, y) of a
// plane is the reconstruction at (x * vis_w / dst_w, y * vis_h / dst_h),
// rounded down. One thread per target sample; grid.y = plane.
//
// Exact-half colour planes (dst = vis / 2 on both axes) follow the reference's
// 4x4 block store (color_store.h:538-559, transform_avx2.c:528-570): a block
// of nx x ny target samples computes only the first nx*ny entries of a 4-wide
// row-major sample array and then reads entry iy*4 + ix, so in a right-edge
// block narrower than 8 source pixels (nx < 4) the entries at or past nx*ny
// still hold the previous block's samples, the same (ix, iy) one block to the
// left (`half_edge` 1: planes wider than one block, whose edge blocks follow
// their left neighbour in the same slice band). In a plane one block wide the
// previous block is the one above in the same band: its entries below 4 * nx
// were written, so a partial last block row whose band also holds the row
// above reads those (`half_edge` 2), and every entry no block of the band
// wrote is delivered as a zero residual, the mid-level sample (`half_edge` 3:
// the last block row starts its own band).
struct DecimPlane {
    uint64_t src_off, dst_off;
    uint32_t vis_w, vis_h, dst_w, dst_h;
    uint32_t half_edge, mid;
};

__global__ void __launch_bounds__(256) k_decimate(const DecimPlane* __restrict__ dp, uint16_t* __restrict__ out)
{
    const DecimPlane P = dp[blockIdx.y];
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)P.dst_w * P.dst_h) { return; }
    const uint32_t ty = (uint32_t)(i / P.dst_w), tx = (uint32_t)(i % P.dst_w);
    uint32_t sx = (uint32_t)(((uint64_t)tx * P.vis_w) / P.dst_w);
    uint32_t sy = (uint32_t)(((uint64_t)ty * P.vis_h) / P.dst_h);
    if (P.half_edge != 0u) {
        const uint32_t px0 = (tx >> 2) * 8u, py0 = (ty >> 2) * 8u;
        const uint32_t nx = min(8u, P.vis_w - px0) / 2u;
        const uint32_t ny = min(8u, P.vis_h - py0) / 2u;
        const uint32_t k = (ty & 3u) * 4u + (tx & 3u);
        if (nx < 4u && k >= nx * ny) {
            if (P.half_edge == 1u) {
                sx -= 8u;               // px0 >= 8: not the first block column
            } else if (P.half_edge == 2u && ny < 4u && k < 4u * nx) {
                sy -= 8u;               // the partial last row, below row 0
            } else {
                out[P.dst_off + i] = (uint16_t)P.mid;
                return;
            }
        }
    }
    out[P.dst_off + i] = out[P.src_off + (uint64_t)sy * P.vis_w + sx];
}

// ------------------------------------------------------------------ alpha

struct BitR {
    const uint8_t* d;
    uint64_t nbits, pos;
};

__device__ __forceinline__ bool br_bit(BitR& r, uint32_t& b)
{
    if (r.pos >= r.nbits) { return false; }
    b = (__ldg(r.d + (r.pos >> 3)) >> (7u - (uint32_t)(r.pos & 7u))) & 1u;
    r.pos++;
    return true;
}

__device__ inline int32_t rice_get(BitR& r, uint32_t k, uint32_t mmax, uint32_t& m)
{
    uint32_t q = 0, b = 0;
    while (q < 31u) {
        if (!br_bit(r, b)) { return TCG_ERR_TRUNCATED; }
        if (b == 0u) { break; }
        ++q;
    }
    uint64_t v;
    if (q == 31u) {
        if (r.nbits - r.pos < 32u) { return TCG_ERR_TRUNCATED; }
        uint32_t lit = 0;
        for (int i = 0; i < 32; ++i) { br_bit(r, b); lit = (lit << 1) | b; }
        v = lit;
    } else {
        if (r.nbits - r.pos < k) { return TCG_ERR_TRUNCATED; }
        uint32_t rem = 0;
        for (uint32_t i = 0; i < k; ++i) { br_bit(r, b); rem = (rem << 1) | b; }
        v = ((uint64_t)q << k) | rem;
    }
    if (v > mmax) { return TCG_ERR_MALFORMED; }
    m = (uint32_t)v;
    return 0;
}

__global__ void k_dalpha(const DSlice* __restrict__ slices, const uint32_t* __restrict__ aslices, uint32_t na,
                         const DPlane* __restrict__ planes, const uint8_t* __restrict__ pkt, int32_t* __restrict__ res,
                         int32_t* __restrict__ status)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= na) { return; }
    const uint32_t si = aslices[i];
    if (status[si] != 0) { return; }
    const DSlice& S = slices[si];
    const DPlane& P = planes[S.plane];
    const uint64_t count = (uint64_t)P.coded_w * S.bh * 8u;
    int32_t* rr = res + S.res_off;
    BitR r = {pkt + S.pay, (uint64_t)S.size * 8u, 0};
    int32_t rc = 0;
    uint64_t pos = 0;
    while (pos < count) {
        const uint64_t remaining = count - pos;
        uint32_t run, lv;
        if ((rc = rice_get(r, S.k2, (uint32_t)remaining, run)) != 0) { break; }
        if ((rc = rice_get(r, S.k1, 0x00020000u, lv)) != 0) { break; }
        if (lv == 0u) {
            if ((uint64_t)run != remaining) { rc = TCG_ERR_MALFORMED; }
            break;
        }
        if ((uint64_t)run + 1u > remaining) { rc = TCG_ERR_MALFORMED; break; }
        rr[pos + run] = unmap_s(lv);
        pos += (uint64_t)run + 1u;
    }
    if (rc == 0) {
        const uint64_t p = (r.pos + 7u) & ~(uint64_t)7u;
        if (p > r.nbits) { rc = TCG_ERR_TRUNCATED; }
        else if (p != r.nbits) { rc = TCG_ERR_MALFORMED; }
    }
    status[si] = rc;
}

// Anti-diagonal wavefront over one band, in groups of 128 rows: thread t owns
// group row t and at step d reconstructs column x = d - t from its left value,
// the row above (shared memory, double buffered) and the above-left value kept
// from the previous step. The first row of a group reads the previous group's
// last row from `edge` (dynamic shared memory, coded_w entries), which the
// group's last row overwrites 127 columns behind the readers.
__global__ void __launch_bounds__(128) k_dalpha_med(const DSlice* __restrict__ slices, const uint32_t* __restrict__ aslices,
                                                    const DPlane* __restrict__ planes, const int32_t* __restrict__ res,
                                                    int32_t* __restrict__ status, uint16_t* __restrict__ out)
{
    extern __shared__ int32_t edge[];
    __shared__ int32_t line[2][128];
    __shared__ int32_t bad;
    const uint32_t si = aslices[blockIdx.x];
    if (status[si] != 0) { return; }
    const DSlice& S = slices[si];
    const DPlane& P = planes[S.plane];
    const uint32_t H = S.bh * 8u, W = P.coded_w;
    const uint32_t t = threadIdx.x;
    const uint32_t mask = P.alpha_shift ? ((1u << P.alpha_shift) - 1u) : 0u;
    const int32_t* rr = res + S.res_off;
    if (t == 0) { bad = 0; }
    __syncthreads();
    for (uint32_t g0 = 0; g0 < H; g0 += 128u) {
        const uint32_t gh = min(128u, H - g0);
        const uint32_t y = g0 + t;          // band row
        const uint32_t gy = S.y0 * 8u + y;  // plane row
        int32_t left = 0, upleft = 0;
        for (uint32_t d = 0; d < W + gh - 1u; ++d) {
            const uint32_t b = d & 1u;
            if (t < gh && d >= t && d - t < W) {
                const uint32_t x = d - t;
                int32_t up = 0;
                if (y > 0u) { up = t > 0u ? line[b ^ 1u][t - 1u] : edge[x]; }
                int32_t pred;
                if (y == 0u) { pred = x == 0u ? 0 : left; }
                else if (x == 0u) { pred = up; }
                else if (upleft >= left && upleft >= up) { pred = left < up ? left : up; }
                else if (upleft <= left && upleft <= up) { pred = left < up ? up : left; }
                else { pred = left + up - upleft; }
                int32_t v = pred + rr[(size_t)y * W + x];
                v = v < 0 ? 0 : (v > 65535 ? 65535 : v);
                if (mask != 0u && ((uint32_t)v & mask) != 0u) { bad = 1; }
                if (gy < P.vis_h && x < P.vis_w) { out[P.out_off + (size_t)gy * P.vis_w + x] = (uint16_t)v; }
                line[b][t] = v;
                if (t == gh - 1u) { edge[x] = v; }
                left = v;
                upleft = up;
            }
            __syncthreads();
        }
    }
    if (t == 0 && bad) { status[si] = TCG_ERR_MALFORMED; }
}

// ------------------------------------------------------------------ concealment

__global__ void __launch_bounds__(256) k_dconceal(const DSlice* __restrict__ slices, const DPlane* __restrict__ planes,
                                                  const int32_t* __restrict__ status, uint16_t* __restrict__ out)
{
    const uint32_t si = blockIdx.x;
    if (status[si] == 0) { return; }
    const DSlice& S = slices[si];
    const DPlane& P = planes[S.plane];
    const uint16_t fill = P.kind == TCG_PLANE_ALPHA ? 0xFFFFu : (uint16_t)(1u << (P.bd - 1u));
    const uint32_t y0 = S.y0 * 8u;
    const uint32_t rows = min(S.bh * 8u, P.vis_h - y0);
    const uint64_t n = (uint64_t)rows * P.vis_w;
    uint16_t* dst = out + P.out_off + (size_t)y0 * P.vis_w;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) { dst[i] = fill; }
}

// ------------------------------------------------------------------ deblock

struct DbPlane {
    uint64_t off;
    uint32_t w, h, alpha, beta, clip, maxv;
    uint32_t unit;      // edge grid: 8 at full size, 4 on an exact half
};

__device__ __forceinline__ bool db_gate(int32_t p1, int32_t p0, int32_t q0, int32_t q1, int32_t a, int32_t b)
{
    return (uint32_t)abs(q0 - p0) < (uint32_t)a && (uint32_t)abs(p1 - p0) < (uint32_t)b && (uint32_t)abs(q1 - q0) < (uint32_t)b;
}

__device__ __forceinline__ int32_t db_delta(int32_t p1, int32_t p0, int32_t q0, int32_t q1, int32_t clip)
{
    int32_t d = (12 * (q0 - p0) + 4 * (p1 - q1) + 8) >> 4;
    const int32_t dl = q0 - p0;
    const int32_t half = dl >= 0 ? (dl >> 1) : -((-dl) >> 1);
    if (half >= 0) { d = d > half ? half : d; d = d < 0 ? 0 : d; }
    else { d = d < half ? half : d; d = d > 0 ? 0 : d; }
    return d < -clip ? -clip : (d > clip ? clip : d);
}

__device__ __forceinline__ void db_apply(uint16_t* a, uint16_t* b, uint16_t* c, uint16_t* e, int32_t p1, int32_t p0,
                                         int32_t q0, int32_t q1, int32_t d, int32_t maxv)
{
    auto cl = [maxv](int32_t v) { return (uint16_t)(v < 0 ? 0 : (v > maxv ? maxv : v)); };
    *b = cl(p0 + d);
    *c = cl(q0 - d);
    *a = cl(p1 + (d >> 1));
    *e = cl(q1 - (d >> 1));
}

// vertical edges: one thread per (row, edge)
__global__ void k_deblock_v(const DbPlane* __restrict__ dp, uint32_t np, uint16_t* __restrict__ out)
{
    const DbPlane P = dp[blockIdx.y];
    const uint32_t edges = P.w / P.unit - 1u;
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)edges * P.h) { return; }
    const uint32_t y = (uint32_t)(i / edges), x0 = P.unit * (uint32_t)(i % edges + 1u);
    uint16_t* r = out + P.off + (size_t)y * P.w;
    const int32_t p1 = r[x0 - 2], p0 = r[x0 - 1], q0 = r[x0], q1 = r[x0 + 1];
    if (db_gate(p1, p0, q0, q1, (int32_t)P.alpha, (int32_t)P.beta)) {
        db_apply(r + x0 - 2, r + x0 - 1, r + x0, r + x0 + 1, p1, p0, q0, q1, db_delta(p1, p0, q0, q1, (int32_t)P.clip),
                 (int32_t)P.maxv);
    }
    (void)np;
}

// horizontal edges: one thread per (edge row, column)
__global__ void k_deblock_h(const DbPlane* __restrict__ dp, uint32_t np, uint16_t* __restrict__ out)
{
    const DbPlane P = dp[blockIdx.y];
    const uint32_t edges = P.h / P.unit - 1u;
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)edges * P.w) { return; }
    const uint32_t r = (uint32_t)(i / P.w) + 1u, x = (uint32_t)(i % P.w);
    const uint32_t y0 = P.unit * r;
    uint16_t* b = out + P.off + x;
    uint16_t* a2 = b + (size_t)(y0 - 2u) * P.w;
    uint16_t* a1 = b + (size_t)(y0 - 1u) * P.w;
    uint16_t* b0 = b + (size_t)y0 * P.w;
    uint16_t* b1 = b + (size_t)(y0 + 1u) * P.w;
    const int32_t p1 = *a2, p0 = *a1, q0 = *b0, q1 = *b1;
    if (db_gate(p1, p0, q0, q1, (int32_t)P.alpha, (int32_t)P.beta)) {
        db_apply(a2, a1, b0, b1, p1, p0, q0, q1, db_delta(p1, p0, q0, q1, (int32_t)P.clip), (int32_t)P.maxv);
    }
    (void)np;
}

// ------------------------------------------------------------------ driver

static size_t align_up(size_t v, size_t a) { return (v + a - 1u) / a * a; }

static uint32_t host_qp_scale(uint32_t refined, uint32_t qp)
{
    static const uint32_t s[64] = {
        1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4, 5, 6, 7, 8, 10, 11, 13, 16, 19, 23, 27, 32, 38, 45, 54, 64, 76, 91, 108,
        128, 152, 181, 215, 256, 304, 362, 431, 512, 609, 724, 861, 1024, 1218, 1448, 1722,
        2048, 2435, 2896, 3444, 4096, 4871, 5793, 6889, 8192, 9742, 11585, 13777, 16384, 19484, 23170, 27555};
    static const uint32_t hi[2][32] = {
        {32768, 38968, 46341, 55109, 65536, 77936, 92682, 110218, 131072, 155872, 185364, 220436, 262144, 311744, 370728,
         440872, 524288, 623487, 741455, 881744, 1048576, 1246974, 1482910, 1763488, 2097152, 2493948, 2965821, 3526975,
         4194304, 4987896, 5931642, 7053950},
        {32768, 36781, 41285, 46341, 52016, 58386, 65536, 73562, 82570, 92682, 104032, 116772, 131072, 147123, 165140,
         185364, 208064, 233544, 262144, 294247, 330281, 370728, 416128, 467088, 524288, 588493, 660561, 741455, 832255,
         934175, 1048576, 1176987}};
    return qp < 64u ? s[qp] : hi[refined ? 1 : 0][qp - 64u];
}

// --------------------------------------------------------- decode-chain tuner
//
// lane-tiling instantiations (named so the launch macro sees one argument)
#define K_DCHAIN_L8 k_dchain<8>
#define K_DCHAIN_L4 k_dchain<4>
#define K_DCHAIN_L2 k_dchain<2>
#define K_DCHAIN_L1 k_dchain<1>

// Tilings of the slice decode: one lane per slice with 8, 4, 2 or 1 slices
// per warp (more slices per warp cost fewer issue slots, fewer cost less
// divergence on each lane's chain), and one warp per slice (lanes hold the
// alphabet; most issue slots). The first batch of each size class (by log2 of
// the colour-slice count) runs the tilings that can win and keeps the fastest:
// 1, 2 and 4 slices per warp (one per warp when the GPU has room for every
// chain, more when the chains compete for issue slots), and a split where the
// largest slices (half of the batch's blocks) run one per warp while the rest
// run four per warp on a second stream, so the short chains take fewer issue
// slots from the long ones that set the batch time.
// TCG_DCHAIN=lane|lane4|lane2|lane1|warp|split forces any one ("lane" is 8).
enum DchainTiling { DCH_TILE_LANE = 0, DCH_TILE_WARP = 1, DCH_TILE_LANE4 = 2, DCH_TILE_LANE2 = 3, DCH_TILE_LANE1 = 4,
                    DCH_TILE_SPLIT = 5 };

static std::mutex g_tune_mu;
static int8_t g_tune[33] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                            -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};

static int dchain_forced()
{
    const char* v = getenv("TCG_DCHAIN");
    if (v == nullptr) { return -1; }
    if (strcmp(v, "lane") == 0) { return DCH_TILE_LANE; }
    if (strcmp(v, "lane4") == 0) { return DCH_TILE_LANE4; }
    if (strcmp(v, "lane2") == 0) { return DCH_TILE_LANE2; }
    if (strcmp(v, "lane1") == 0) { return DCH_TILE_LANE1; }
    if (strcmp(v, "warp") == 0) { return DCH_TILE_WARP; }
    if (strcmp(v, "split") == 0) { return DCH_TILE_SPLIT; }
    return -1;
}

static uint32_t size_class(uint32_t nc) { return nc == 0u ? 0u : 32u - (uint32_t)__builtin_clz(nc); }

extern "C" __attribute__((visibility("default"))) int32_t tcg_dchain_tiling(uint32_t nc)
{
    const int f = dchain_forced();
    if (f >= 0) { return f; }
    std::lock_guard<std::mutex> g(g_tune_mu);
    return g_tune[size_class(nc)];
}

// What decode_outputs and decode_finish need of a launched batch.
struct DecPending {
    std::vector<uint32_t> frame_slice0;  // each frame's first entry in slice_map
    std::vector<int32_t> slice_map;      // device slice of every packet slice (-1: not decoded)
    std::vector<DPlane> planes;          // output offsets and sizes, frames in order
    uint32_t ns = 0;                     // slices
};

// Enqueue one batch on the context's streams: descriptors, packet copies and
// kernels. The packet copies start after `after` (when given) and C->gate is
// recorded behind them. load_nc: colour slices of the whole pipelined batch
// this one is a chunk of (0: the batch is decoded alone).
static int32_t decode_launch(Ctx* C, const tcg_dec_frame* frames, uint32_t count, cudaEvent_t after,
                             uint32_t load_nc, DecPending& pend)
{
    std::vector<uint32_t>& frame_slice0 = pend.frame_slice0;
    std::vector<DPlane>& planes = pend.planes;
    planes.clear();
    pend.slice_map.clear();
    std::vector<DSlice> slices;
    std::vector<uint32_t> cslices, aslices, slice_tab;
    std::vector<DbPlane> dbp;
    std::vector<DecimPlane> decim;
    std::vector<uint64_t> pkt_off(count, 0);
    frame_slice0.assign(count, 0u);
    uint64_t out_elems = 0, pkt_bytes = 0, nblk = 0, alpha_res = 0;
    uint32_t max_cols = 1;
    for (uint32_t f = 0; f < count; ++f) {
        const tcg_dec_frame& F = frames[f];
        frame_slice0[f] = (uint32_t)pend.slice_map.size();
        if (F.skip) { continue; }
        pkt_off[f] = pkt_bytes;
        pkt_bytes = align_up(pkt_bytes + F.size, 256);
        const uint32_t pg0 = (uint32_t)planes.size();
        for (uint32_t p = 0; p < F.planes; ++p) {
            DPlane P;
            memset(&P, 0, sizeof(P));
            P.out_off = out_elems;
            out_elems = align_up(out_elems + (uint64_t)F.vis_w[p] * F.vis_h[p], 64);
            P.vis_w = F.vis_w[p]; P.vis_h = F.vis_h[p]; P.coded_w = F.coded_w[p];
            P.cols = F.cols[p]; P.rows = F.rows[p];
            P.bd = F.bit_depth;
            P.kind = (p == 3u && F.alpha_mode != 0u) ? TCG_PLANE_ALPHA : TCG_PLANE_COLOR;
            P.alpha_shift = P.kind == TCG_PLANE_ALPHA ? F.alpha_shift : 0u;
            P.refined = F.refined;
            P.blk0 = (uint32_t)nblk;
            P.frame = f;
            P.climit = F.climit;
            memcpy(P.qm, F.qm[p], sizeof(P.qm));
            if (F.scaled) {
                // the delivered plane follows its reconstruction in the same buffer
                P.dst_off = out_elems;
                P.dst_w = F.dst_w[p];
                P.dst_h = F.dst_h[p];
                out_elems = align_up(out_elems + (uint64_t)P.dst_w * P.dst_h, 64);
                const bool half = P.kind == TCG_PLANE_COLOR && (uint64_t)P.dst_w * 2u == P.vis_w &&
                                  (uint64_t)P.dst_h * 2u == P.vis_h;
                uint32_t half_edge = half ? (P.vis_w > 8u ? 1u : 2u) : 0u;
                if (half_edge == 2u) {
                    const uint32_t last = (P.vis_h - 1u) / 8u;  // last block row
                    bool own = last == 0u;
                    for (uint32_t i = 0; i < F.slices && !own; ++i) {
                        own = F.slice[i].plane == p && F.slice[i].y0 == last;
                    }
                    half_edge = own ? 3u : 2u;
                }
                DecimPlane dm = {P.out_off, P.dst_off, P.vis_w, P.vis_h, P.dst_w, P.dst_h, half_edge,
                                 1u << (P.bd - 1u)};
                if (P.dst_w > 0u && P.dst_h > 0u) { decim.push_back(dm); }
            } else {
                P.dst_off = P.out_off;
                P.dst_w = P.vis_w;
                P.dst_h = P.vis_h;
            }
            if (P.kind == TCG_PLANE_COLOR) { nblk += (uint64_t)P.cols * P.rows; }
            max_cols = P.cols > max_cols ? P.cols : max_cols;
            planes.push_back(P);
            const uint32_t u = F.db_unit;
            if (u != 0u && p < 3u) {
                // deblocking of the delivered plane (reference deblock.c:305-329)
                const uint32_t w = P.dst_w, h = P.dst_h;
                if (w >= 2u * u && h >= 2u * u && (w % u) == 0u && (h % u) == 0u && F.qp_base <= 95u) {
                    const uint32_t sc = host_qp_scale(F.refined, F.qp_base);
                    uint32_t step = (sc * 3u + 173056u / 2u) / 173056u;
                    step = step < 1u ? 1u : step;
                    uint32_t a = step * 2u;
                    a = a < 3u ? 3u : (a > 48u ? 48u : a);
                    DbPlane d = {P.dst_off, w, h, a, a / 2u + 2u, a >> 1, (1u << F.bit_depth) - 1u, u};
                    dbp.push_back(d);
                }
            }
        }
        for (uint32_t i = 0; i < F.slices; ++i) {
            const tcg_dec_slice& I = F.slice[i];
            if (I.plane >= F.planes) {  // a plane not delivered (dropped alpha)
                pend.slice_map.push_back(-1);
                continue;
            }
            pend.slice_map.push_back((int32_t)slices.size());
            DSlice S;
            memset(&S, 0, sizeof(S));
            const DPlane& P = planes[pg0 + I.plane];
            S.frame = f; S.plane = pg0 + I.plane; S.pidx = I.plane; S.kind = P.kind;
            S.y0 = I.y0; S.bh = I.bh; S.cols = P.cols;
            S.size = I.size; S.crc = I.crc; S.qp = I.qp; S.k1 = I.k1; S.k2 = I.k2;
            S.pay = pkt_off[f] + I.off;
            const uint32_t si = (uint32_t)slices.size();
            if (S.kind == TCG_PLANE_COLOR) {
                S.blk0 = P.blk0 + I.y0 * P.cols;
                S.nblk = I.bh * P.cols;
                slice_tab.push_back((uint32_t)cslices.size());
                cslices.push_back(si);
            } else {
                S.res_off = alpha_res;
                alpha_res += (uint64_t)P.coded_w * I.bh * 8u;
                slice_tab.push_back(0u);
                aslices.push_back(si);
            }
            slices.push_back(S);
        }
    }
    const uint32_t ns = (uint32_t)slices.size(), nc = (uint32_t)cslices.size(), na = (uint32_t)aslices.size();
    const size_t desc = align_up(planes.size() * sizeof(DPlane), 256) + align_up(ns * sizeof(DSlice), 256) +
                        align_up((size_t)(nc + na) * 4u + 16, 256) + align_up((size_t)ns * 4u + 16, 256) +
                        align_up(dbp.size() * sizeof(DbPlane) + 16, 256) +
                        align_up((size_t)nc * 4u + 16, 256) + align_up(decim.size() * sizeof(DecimPlane) + 16, 256) +
                        align_up((size_t)nc * 4u + 16, 256);
    if (!dreserve(C, B_DEC_PKT, pkt_bytes + 256) || !dreserve(C, B_DEC_COEF, nblk * 256u + 256) ||
        !dreserve(C, B_UMAP, (nblk + 31u) / 32u * 4u + 256) ||
        !dreserve(C, B_DEC_TAB, (size_t)nc * DTAB_BYTES + 256) || !dreserve(C, B_DEC_OUT, out_elems * 2u + 256) ||
        !dreserve(C, B_DEC_RES, (size_t)ns * 4u + 256) || !dreserve(C, B_ALPHA, alpha_res * 4u + 256) ||
        !dreserve(C, B_DESC, desc + 256) || !hreserve(C, 0, desc + 256) || !hreserve(C, 1, (size_t)ns * 4u + 256)) {
        return TCG_ERR_OUT_OF_MEMORY;
    }
    cudaStream_t st = C->stream;
    uint8_t* hd = (uint8_t*)C->h[0].p;
    uint8_t* dd = dptr<uint8_t>(C, B_DESC);
    size_t o = 0;
    auto put = [&](const void* src, size_t n) -> size_t {
        const size_t at = o;
        if (n) { memcpy(hd + o, src, n); }
        o = align_up(o + n, 256);
        return at;
    };
    std::vector<uint32_t> cs_as(cslices);
    cs_as.insert(cs_as.end(), aslices.begin(), aslices.end());
    // chain lanes: largest slices first so a block's lanes finish together
    std::vector<uint32_t> ord(cslices);
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return slices[a].nblk > slices[b].nblk; });
    const size_t o_pl = put(planes.data(), planes.size() * sizeof(DPlane));
    const size_t o_sl = put(slices.data(), ns * sizeof(DSlice));
    const size_t o_ca = put(cs_as.data(), cs_as.size() * 4u);
    const size_t o_st = put(slice_tab.data(), slice_tab.size() * 4u);
    const size_t o_db = put(dbp.data(), dbp.size() * sizeof(DbPlane));
    const size_t o_or = put(ord.data(), ord.size() * 4u);
    const size_t o_dm = put(decim.data(), decim.size() * sizeof(DecimPlane));
    std::vector<uint32_t> cstart(nc);  // first block of each colour slice, for the reconstruction's unit lookup
    for (uint32_t i = 0; i < nc; ++i) { cstart[i] = slices[cslices[i]].blk0; }
    const size_t o_cb = put(cstart.data(), (size_t)nc * 4u);
    TCG_CHECK(cudaMemcpyAsync(dd, hd, o, cudaMemcpyHostToDevice, st));
    const DPlane* d_pl = (const DPlane*)(dd + o_pl);
    const DSlice* d_sl = (const DSlice*)(dd + o_sl);
    const uint32_t* d_cs = (const uint32_t*)(dd + o_ca);
    const uint32_t* d_as = d_cs + nc;
    const uint32_t* d_st = (const uint32_t*)(dd + o_st);
    const DbPlane* d_db = (const DbPlane*)(dd + o_db);
    const uint32_t* d_ord = (const uint32_t*)(dd + o_or);
    const DecimPlane* d_dm = (const DecimPlane*)(dd + o_dm);
    const uint32_t* d_cb = (const uint32_t*)(dd + o_cb);
    uint8_t* d_pkt = dptr<uint8_t>(C, B_DEC_PKT);
    call_begin(C);
    if (after != nullptr) { TCG_CHECK(cudaStreamWaitEvent(st, after, 0)); }
    for (uint32_t f = 0; f < count; ++f) {
        if (frames[f].skip) { continue; }
        TCG_CHECK(cudaMemcpyAsync(d_pkt + pkt_off[f], frames[f].packet, frames[f].size, cudaMemcpyDefault, st));
    }
    TCG_CHECK(cudaEventRecord(C->gate, st));
    int32_t* d_status = dptr<int32_t>(C, B_DEC_RES);
    int32_t* d_coef = dptr<int32_t>(C, B_DEC_COEF);
    uint8_t* d_tab = dptr<uint8_t>(C, B_DEC_TAB);
    uint16_t* d_out = dptr<uint16_t>(C, B_DEC_OUT);
    int32_t* d_ares = dptr<int32_t>(C, B_ALPHA);
    const DevTables& T = tables();
    if (ns > 0) {
        TCG_CHECK(cudaMemsetAsync(d_status, 0, (size_t)ns * 4u, st));
        TCG_LAUNCH(C, K_DCRC, k_dcrc, ns, 256, 0, d_sl, d_pkt, T.crc, d_status);
    }
    if (na > 0) {
        // Alpha slices (Rice run/level decode, then MED reconstruction) share no
        // slice, status entry or output plane with the colour slices, so they
        // run on a third stream beside the colour chain; the stream rejoins
        // before concealment.
        cudaStream_t as = aux_stream(C);
        if (as == nullptr) { return TCG_ERR_OUT_OF_MEMORY; }
        TCG_CHECK(cudaEventRecord(C->afork, st));
        TCG_CHECK(cudaStreamWaitEvent(as, C->afork, 0));
        TCG_CHECK(cudaMemsetAsync(d_ares, 0, alpha_res * 4u, as));
        TCG_LAUNCH_ON(C, as, K_DALPHA, k_dalpha, (na + 63u) / 64u, 64, 0, d_sl, d_as, na, d_pl, d_pkt, d_ares,
                      d_status);
        uint32_t max_w = 8;
        for (uint32_t a : aslices) { max_w = std::max(max_w, planes[slices[a].plane].coded_w); }
        const size_t esmem = (size_t)max_w * 4u;
        static size_t eattr = 0;
        if (esmem > eattr) {
            cudaFuncSetAttribute(k_dalpha_med, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esmem);
            eattr = esmem;
        }
        TCG_LAUNCH_ON(C, as, K_DALPHA_MED, k_dalpha_med, na, 128, esmem, d_sl, d_as, d_pl, d_ares, d_status, d_out);
        TCG_CHECK(cudaEventRecord(C->ajoin, as));
    }
    if (nc > 0) {
        TCG_LAUNCH(C, K_DTABLES, k_dtables, nc, 32, 0, d_sl, d_cs, d_pl, d_pkt, T.qscale, d_tab, d_status);
        static bool attr = false;
        if (!attr) {
            TCG_CHECK(cudaFuncSetAttribute(k_dchain<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dch_smem(8)));
            TCG_CHECK(cudaFuncSetAttribute(k_dchain<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dch_smem(4)));
            attr = true;
        }
        const size_t wsmem = (size_t)max_cols * 8u;  // two DC rows per slice (warp tiling)
        // split point: the largest slices (in chain order) up to half of the blocks
        uint32_t nsplit = 0;
        {
            uint64_t tot = 0, acc = 0;
            for (uint32_t si : ord) { tot += slices[si].nblk; }
            while (nsplit < nc && 2u * acc < tot) { acc += slices[ord[nsplit++]].nblk; }
        }
        auto run = [&](int tiling) -> int32_t {
            switch (tiling) {
            case DCH_TILE_SPLIT: {
                cudaStream_t sd = side_stream(C);
                if (sd == nullptr) { return TCG_ERR_OUT_OF_MEMORY; }
                TCG_CHECK(cudaMemsetAsync(d_coef, 0, nblk * 256u, st));
                tcg::kern_begin(C, K_DCHAIN);
                TCG_CHECK(cudaEventRecord(C->fork, st));
                TCG_CHECK(cudaStreamWaitEvent(sd, C->fork, 0));
                k_dchain<1><<<nsplit, 32, dch_smem(1), st>>>(d_sl, d_ord, nsplit, d_st, d_pl, d_pkt, d_tab, d_coef,
                                                               d_status);
                if (nc > nsplit) {
                    k_dchain<4><<<(nc - nsplit + 3u) / 4u, 32, dch_smem(4), sd>>>(
                        d_sl, d_ord + nsplit, nc - nsplit, d_st, d_pl, d_pkt, d_tab, d_coef, d_status);
                }
                tcg::note_launch(nc > nsplit ? 2u : 1u);
                TCG_CHECK(cudaGetLastError());
                TCG_CHECK(cudaEventRecord(C->join, sd));
                TCG_CHECK(cudaStreamWaitEvent(st, C->join, 0));
                tcg::kern_end(C);
                if (tcg::sync_each()) { TCG_CHECK(cudaStreamSynchronize(st)); }
                return TCG_OK;
            }
            case DCH_TILE_WARP:
                // the warp tiling writes every coefficient of the blocks it decodes
                TCG_LAUNCH(C, K_DCHAIN_W, k_dchain_w, nc, 32, wsmem, d_sl, d_cs, d_pl, d_pkt, d_tab, d_coef, d_status);
                return TCG_OK;
            case DCH_TILE_LANE4:
                TCG_CHECK(cudaMemsetAsync(d_coef, 0, nblk * 256u, st));
                TCG_LAUNCH(C, K_DCHAIN, K_DCHAIN_L4, (nc + 3u) / 4u, 32, dch_smem(4), d_sl, d_ord, nc, d_st, d_pl,
                           d_pkt, d_tab, d_coef, d_status);
                return TCG_OK;
            case DCH_TILE_LANE2:
                TCG_CHECK(cudaMemsetAsync(d_coef, 0, nblk * 256u, st));
                TCG_LAUNCH(C, K_DCHAIN, K_DCHAIN_L2, (nc + 1u) / 2u, 32, dch_smem(2), d_sl, d_ord, nc, d_st, d_pl,
                           d_pkt, d_tab, d_coef, d_status);
                return TCG_OK;
            case DCH_TILE_LANE1:
                TCG_CHECK(cudaMemsetAsync(d_coef, 0, nblk * 256u, st));
                TCG_LAUNCH(C, K_DCHAIN, K_DCHAIN_L1, nc, 32, dch_smem(1), d_sl, d_ord, nc, d_st, d_pl, d_pkt, d_tab,
                           d_coef, d_status);
                return TCG_OK;
            default:
                TCG_CHECK(cudaMemsetAsync(d_coef, 0, nblk * 256u, st));
                TCG_LAUNCH(C, K_DCHAIN, K_DCHAIN_L8, (nc + 7u) / 8u, 32, dch_smem(8), d_sl, d_ord, nc, d_st, d_pl,
                           d_pkt, d_tab, d_coef, d_status);
                return TCG_OK;
            }
        };
        // A chunk of a pipelined batch decodes beside the other chunks: it takes
        // the tiling chosen for the whole batch's slice count (the split when
        // none is chosen yet) and is never timed alone.
        int tiling = dchain_forced();
        const uint32_t cls = size_class(load_nc != 0u ? load_nc : nc);
        if (tiling < 0) {
            std::lock_guard<std::mutex> g(g_tune_mu);
            tiling = g_tune[cls];
        }
        if (tiling < 0 && load_nc != 0u) { tiling = DCH_TILE_SPLIT; }
        if (tiling >= 0) {
            const int32_t rc = run(tiling);
            if (rc != TCG_OK) { return rc; }
        } else {
            // each candidate decodes the whole batch once, timed on the stream; the
            // last run's output stands (all tilings write identical results)
            constexpr int cand[4] = {DCH_TILE_SPLIT, DCH_TILE_LANE4, DCH_TILE_LANE2, DCH_TILE_LANE1};
            cudaEvent_t e[5];
            for (auto& x : e) { TCG_CHECK(cudaEventCreate(&x)); }
            int32_t rc = cudaEventRecord(e[0], st) == cudaSuccess ? TCG_OK : cuda_fail(cudaGetLastError(), "tuner");
            for (int k = 0; k < 4 && rc == TCG_OK; ++k) {
                rc = run(cand[k]);
                if (rc == TCG_OK && cudaEventRecord(e[k + 1], st) != cudaSuccess) {
                    rc = cuda_fail(cudaGetLastError(), "tuner");
                }
            }
            if (rc == TCG_OK && cudaEventSynchronize(e[4]) != cudaSuccess) { rc = cuda_fail(cudaGetLastError(), "tuner"); }
            if (rc != TCG_OK) {
                for (auto& x : e) { cudaEventDestroy(x); }
                return rc;
            }
            int best = cand[0];
            float best_ms = 0.f;
            for (int k = 0; k < 4; ++k) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e[k], e[k + 1]);
                if (k == 0 || ms < best_ms) { best = cand[k]; best_ms = ms; }
            }
            for (auto& x : e) { cudaEventDestroy(x); }
            std::lock_guard<std::mutex> g(g_tune_mu);
            g_tune[cls] = (int8_t)best;
        }
        uint32_t* d_umap = dptr<uint32_t>(C, B_UMAP);
        TCG_LAUNCH(C, K_UNIT_MAP, k_unit_map, (uint32_t)((nblk + 8191u) / 8192u), 256, 0, d_cb, 1u, nc, (uint32_t)nblk, d_umap);
        TCG_LAUNCH(C, K_DIDCT, k_didct, (uint32_t)((nblk + RB_BLOCKS - 1u) / RB_BLOCKS), 256, 0, d_sl, d_cs, nc, d_st, d_pl,
                   d_tab, d_coef, d_status, (uint32_t)nblk, d_cb, d_umap, d_out);
    }
    if (na > 0) {
        // the alpha planes have been on their own stream since the CRC check
        TCG_CHECK(cudaStreamWaitEvent(st, C->ajoin, 0));
    }
    if (ns > 0) {
        TCG_LAUNCH(C, K_DCONCEAL, k_dconceal, ns, 256, 0, d_sl, d_pl, d_status, d_out);
    }
    if (!decim.empty()) {
        uint64_t mt = 0;
        for (const DecimPlane& d : decim) { mt = std::max<uint64_t>(mt, (uint64_t)d.dst_w * d.dst_h); }
        TCG_LAUNCH(C, K_DECIMATE, k_decimate, dim3((uint32_t)((mt + 255u) / 256u), (uint32_t)decim.size()), 256, 0,
                   d_dm, d_out);
    }
    if (!dbp.empty()) {
        uint64_t mv = 0, mh = 0;
        for (const DbPlane& d : dbp) {
            mv = std::max<uint64_t>(mv, (uint64_t)(d.w / d.unit - 1u) * d.h);
            mh = std::max<uint64_t>(mh, (uint64_t)(d.h / d.unit - 1u) * d.w);
        }
        TCG_LAUNCH(C, K_DEBLOCK_V, k_deblock_v, dim3((uint32_t)((mv + 255u) / 256u), (uint32_t)dbp.size()), 256, 0,
                   d_db, (uint32_t)dbp.size(), d_out);
        TCG_LAUNCH(C, K_DEBLOCK_H, k_deblock_h, dim3((uint32_t)((mh + 255u) / 256u), (uint32_t)dbp.size()), 256, 0,
                   d_db, (uint32_t)dbp.size(), d_out);
    }
    TCG_CHECK(cudaGetLastError());
    pend.ns = ns;
    return 0;
}

// Enqueue the copies of a launched batch's planes to the callers' buffers and
// of its slice statuses to pinned host memory.
static int32_t decode_outputs(Ctx* C, const tcg_dec_frame* frames, const DecPending& pend)
{
    cudaStream_t st = C->stream;
    const std::vector<DPlane>& planes = pend.planes;
    const uint16_t* d_out = dptr<uint16_t>(C, B_DEC_OUT);
    const uint32_t count = (uint32_t)pend.frame_slice0.size();
    uint32_t pg = 0;
    for (uint32_t f = 0; f < count; ++f) {
        const tcg_dec_frame& F = frames[f];
        if (F.skip) { continue; }
        for (uint32_t p = 0; p < F.planes; ++p, ++pg) {
            const DPlane& P = planes[pg];
            if (P.dst_w == 0u || P.dst_h == 0u) { continue; }
            const size_t pitch = (F.dst_stride[p] ? F.dst_stride[p] : P.dst_w) * 2u;
            if (pitch == (size_t)P.dst_w * 2u) {  // tight rows: one flat copy
                TCG_CHECK(cudaMemcpyAsync(F.dst[p], d_out + P.dst_off, pitch * P.dst_h, cudaMemcpyDefault, st));
            } else {
                TCG_CHECK(cudaMemcpy2DAsync(F.dst[p], pitch, d_out + P.dst_off, (size_t)P.dst_w * 2u,
                                            (size_t)P.dst_w * 2u, P.dst_h, cudaMemcpyDefault, st));
            }
        }
    }
    int32_t* hs = (int32_t*)C->h[1].p;
    if (pend.ns > 0) {
        TCG_CHECK(cudaMemcpyAsync(hs, dptr<int32_t>(C, B_DEC_RES), (size_t)pend.ns * 4u, cudaMemcpyDeviceToHost, st));
    }
    return 0;
}

// Wait for a batch whose outputs were enqueued and report each slice's status.
static int32_t decode_finish(Ctx* C, const tcg_dec_frame* frames, const DecPending& pend)
{
    const std::vector<uint32_t>& frame_slice0 = pend.frame_slice0;
    TCG_CHECK(cudaStreamSynchronize(C->stream));
    call_end(C);
    const int32_t* hs = (const int32_t*)C->h[1].p;
    for (uint32_t f = 0; f < (uint32_t)frame_slice0.size(); ++f) {
        const tcg_dec_frame& F = frames[f];
        if (F.skip) { continue; }
        for (uint32_t i = 0; i < F.slices; ++i) {
            const int32_t k = pend.slice_map[frame_slice0[f] + i];
            F.slice_status[i] = (k >= 0 && hs[k] != 0) ? 1u : 0u;
        }
    }
    return 0;
}

static int32_t decode_impl(Ctx* C, const tcg_dec_frame* frames, uint32_t count)
{
    DecPending pend;
    int32_t rc = decode_launch(C, frames, count, nullptr, 0u, pend);
    if (rc == 0) { rc = decode_outputs(C, frames, pend); }
    return rc != 0 ? rc : decode_finish(C, frames, pend);
}

// Host-memory batch in chunks on as many contexts (pipeline_plan): chunk i's
// packet copies queue behind chunk i-1's, so later chunks' packets arrive while
// earlier chunks decode, and earlier chunks' planes go back while later ones
// still decode. Every chunk's packet copies and kernels are enqueued before any
// chunk's output copies, so no upload is queued behind a download that waits
// for kernels. The reported device time spans the first chunk's start to the
// last chunk's end.
static int32_t decode_pipelined(const tcg_dec_frame* frames, const uint32_t* starts, uint32_t k)
{
    Ctx* cs[PIPE_MAX_CHUNKS] = {};
    DecPending fs0[PIPE_MAX_CHUNKS];
    int32_t rc = 0;
    uint32_t launched = 0;
    uint32_t load_nc = 0;  // colour slices of the whole batch
    for (uint32_t f = 0; f < starts[k]; ++f) {
        if (frames[f].skip) { continue; }
        for (uint32_t i = 0; i < frames[f].slices; ++i) {
            load_nc += (frames[f].slice[i].plane == 3u && frames[f].alpha_mode != 0u) ? 0u : 1u;
        }
    }
    for (uint32_t i = 0; i < k && rc == 0; ++i) {
        cs[i] = ctx_acquire();
        if (cs[i] == nullptr) {
            rc = TCG_ERR_NOT_IMPLEMENTED;
            break;
        }
        launched = i + 1u;
        rc = decode_launch(cs[i], frames + starts[i], starts[i + 1] - starts[i], i ? cs[i - 1]->gate : nullptr,
                           std::max(load_nc, 1u), fs0[i]);
    }
    for (uint32_t i = 0; i < launched && rc == 0; ++i) { rc = decode_outputs(cs[i], frames + starts[i], fs0[i]); }
    double span = 0.0;
    for (uint32_t i = 0; i < launched; ++i) {
        if (rc == 0) {
            rc = decode_finish(cs[i], frames + starts[i], fs0[i]);
            if (rc == 0) { span = std::max(span, event_span_ms(cs[0]->t0, cs[i]->t1)); }
        } else {
            cudaStreamSynchronize(cs[i]->stream);
        }
    }
    for (uint32_t i = 0; i < launched; ++i) { ctx_release(cs[i]); }
    if (rc == 0) { set_last_ms(span); }
    return rc;
}

// ------------------------------------------------------------------ packet walk

// One thread per packet: copy the first 61 packet bytes (frame header plus the
// bytes a generation probe inspects) and every slice header reachable inside
// the packet (at most 512), stopping exactly where a host structural parse
// would stop for lack of bytes. Record layout (TCG_WALK_REC in tcg_device.h):
// [64: packet bytes 0..60, zero beyond the packet][u32 walked][u32 end offset]
// [8 pad][512 x 17 slice headers].
constexpr size_t WALK_REC = TCG_WALK_REC;

__global__ void k_walk(const uint8_t* const* __restrict__ pkts, const uint64_t* __restrict__ sizes, uint32_t n,
                       uint8_t* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) { return; }
    const uint8_t* p = pkts[i];
    const uint64_t sz = sizes[i];
    uint8_t* r = out + (size_t)i * WALK_REC;
    for (uint32_t k = 0; k < 64u; ++k) { r[k] = (k < 61u && k < sz) ? p[k] : 0u; }
    uint32_t walked = 0;
    uint64_t off = 53u;
    if (sz >= 53u) {
        uint32_t ns = ((uint32_t)p[30] << 8) | p[31];
        ns = ns > 512u ? 512u : ns;
        for (uint32_t s = 0; s < ns; ++s) {
            if (off > sz || sz - off < 17u) { break; }
            const uint8_t* h = p + off;
            for (uint32_t k = 0; k < 17u; ++k) { r[80u + s * 17u + k] = h[k]; }
            walked = s + 1u;
            off += 17u;
            const uint32_t pay = ((uint32_t)h[0] << 24) | ((uint32_t)h[1] << 16) | ((uint32_t)h[2] << 8) | h[3];
            if (sz - off < pay) { break; }
            off += pay;
        }
    }
    *reinterpret_cast<uint32_t*>(r + 64) = walked;
    *reinterpret_cast<uint32_t*>(r + 68) = (uint32_t)off;
}

static int32_t walk_impl(Ctx* C, const uint8_t* const* pkts, const size_t* sizes, uint32_t n, uint8_t* host_out)
{
    const size_t ptr_bytes = align_up((size_t)n * 8u, 256);
    if (!dreserve(C, B_TMP1, ptr_bytes * 2u + (size_t)n * WALK_REC + 256) || !hreserve(C, 2, ptr_bytes * 2u) ||
        !hreserve(C, 3, (size_t)n * WALK_REC)) {
        return TCG_ERR_OUT_OF_MEMORY;
    }
    uint8_t* hb = (uint8_t*)C->h[2].p;
    memcpy(hb, pkts, (size_t)n * 8u);
    for (uint32_t i = 0; i < n; ++i) { reinterpret_cast<uint64_t*>(hb + ptr_bytes)[i] = sizes[i]; }
    uint8_t* db = dptr<uint8_t>(C, B_TMP1);
    call_begin(C);
    TCG_CHECK(cudaMemcpyAsync(db, hb, ptr_bytes * 2u, cudaMemcpyHostToDevice, C->stream));
    TCG_LAUNCH(C, K_WALK, k_walk, (n + 63u) / 64u, 64, 0, (const uint8_t* const*)db, (const uint64_t*)(db + ptr_bytes),
               n, db + 2u * ptr_bytes);
    TCG_CHECK(cudaMemcpyAsync(C->h[3].p, db + 2u * ptr_bytes, (size_t)n * WALK_REC, cudaMemcpyDeviceToHost, C->stream));
    TCG_CHECK(cudaStreamSynchronize(C->stream));
    call_end(C);
    memcpy(host_out, C->h[3].p, (size_t)n * WALK_REC);
    return 0;
}

// ------------------------------------------------ allocation-free packet walk
//
// Scratch of tcg_walk_packets_noalloc: the packet pointer and size tables and
// one walk record per packet, for at most TCG_NOALLOC_MAX_PACKETS packets. It
// lives in the library's static device data (every GPU that loads the library
// holds these ~550 KB until exit); no call allocates device memory. Host code
// reaches it through the address that cudaGetSymbolAddress reports for the
// current device, looked up on the first call on each device.
constexpr size_t NA_TABLE = (size_t)TCG_NOALLOC_MAX_PACKETS * 8u;
constexpr size_t NA_BYTES = 2u * NA_TABLE + (size_t)TCG_NOALLOC_MAX_PACKETS * WALK_REC;
static __device__ __align__(256) uint8_t g_walk_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
static std::mutex g_na_mu;
static uint8_t* g_na_base[NA_MAX_DEVICES];
static unsigned long long g_na_ctx[NA_MAX_DEVICES];  // context the address belongs to

// Unique id of the calling thread's current context (0 when unknown). A
// context destroyed and created again (cudaDeviceReset, a released primary
// context) gets a new id, so an address looked up in the old one is not reused.
static unsigned long long current_ctx_id()
{
    using get_cur_t = int (*)(void**);
    using get_id_t = int (*)(void*, unsigned long long*);
    static get_cur_t get_cur = nullptr;
    static get_id_t get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            get_cur = reinterpret_cast<get_cur_t>(f);
        }
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            get_id = reinterpret_cast<get_id_t>(f);
        }
        cudaGetLastError();
    });
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur == nullptr || get_id == nullptr || get_cur(&ctx) != 0 || ctx == nullptr || get_id(ctx, &id) != 0) {
        return 0;
    }
    return id;
}

// Device address of the static scratch on the current device, looked up once
// per device and context (the lookup may load the library's device code).
static int32_t noalloc_base(int dev, uint8_t** base)
{
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        tcg_host_set_error(TCG_ERR_LIMIT_EXCEEDED, "allocation-free walk: device ordinal beyond 63");
        return TCG_ERR_LIMIT_EXCEEDED;
    }
    const unsigned long long ctx = current_ctx_id();
    std::lock_guard<std::mutex> g(g_na_mu);
    if (g_na_base[dev] == nullptr || ctx == 0 || g_na_ctx[dev] != ctx) {
        void* p = nullptr;
        TCG_CHECK(cudaGetSymbolAddress(&p, g_walk_scratch));
        g_na_base[dev] = static_cast<uint8_t*>(p);
        g_na_ctx[dev] = ctx;
    }
    *base = g_na_base[dev];
    return 0;
}

// V8 batch decode: the frames' descriptors are concatenated (segments,
// tiles, quantiser steps and planes renumbered into one index space) and
// decoded in one launch sequence: packets and descriptors up, tile CRCs,
// tile tables, chains, reconstruction, planes and per-segment / per-tile
// results back.
static int32_t decode_v8_impl(Ctx* C, const tcg_v8_job* J, uint32_t count)
{
    std::vector<tcg_v8_seg> segs;
    std::vector<tcg_v8_tile> tiles;
    std::vector<uint32_t> q, pinfo;
    std::vector<uint64_t> pkt_off(count), out_off;
    uint64_t pkt_bytes = 0, nblk = 0, out_elems = 0;
    for (uint32_t f = 0; f < count; ++f) {
        const tcg_v8_job& F = J[f];
        pkt_off[f] = pkt_bytes;
        pkt_bytes = align_up(pkt_bytes + F.size, 256);
        const uint32_t seg_base = (uint32_t)segs.size(), tile_base = (uint32_t)tiles.size();
        const uint32_t q_base = (uint32_t)(q.size() / 64u), plane_base = (uint32_t)(pinfo.size() / V8_PINFO);
        const uint32_t sb = 1u << F.sb_log2;
        uint32_t seg0 = seg_base;
        for (uint32_t p = 0; p < 3u; ++p) {
            const uint32_t blocks = F.cols[p] * F.rows[p];
            const uint32_t pi[V8_PINFO] = {(uint32_t)nblk, seg0, F.cols[p], F.vis_w[p], F.vis_h[p],
                                           (uint32_t)(out_elems / 64u), F.sb_log2, F.bit_depth};
            pinfo.insert(pinfo.end(), pi, pi + V8_PINFO);
            out_off.push_back(out_elems);
            nblk += blocks;
            seg0 += (blocks + sb - 1u) / sb;
            out_elems = align_up(out_elems + (uint64_t)F.vis_w[p] * F.vis_h[p], 64);
        }
        for (uint32_t k = 0; k < F.nseg; ++k) {
            tcg_v8_seg g = F.seg[k];
            g.plane += plane_base;
            g.off += (uint32_t)pkt_off[f];
            g.tile = g.tile == UINT32_MAX ? UINT32_MAX : g.tile + tile_base;
            g.qidx += q_base;
            segs.push_back(g);
        }
        for (uint32_t t = 0; t < F.ntile; ++t) {
            tcg_v8_tile T = F.tile[t];
            T.plane += plane_base;
            T.seg0 += seg_base;
            T.table_off += (uint32_t)pkt_off[f];
            T.stream_off += (uint32_t)pkt_off[f];
            tiles.push_back(T);
        }
        q.insert(q.end(), F.q, F.q + (size_t)F.nq * 64u);
    }
    if (pkt_bytes > 0xFFFFFFFFull) {
        tcg_host_set_error(TCG_ERR_LIMIT_EXCEEDED, "V8 batch packets exceed 4 GB: decode fewer frames per call");
        return TCG_ERR_LIMIT_EXCEEDED;
    }
    const uint32_t nseg = (uint32_t)segs.size(), ntile = (uint32_t)tiles.size();
    const uint32_t nplanes = (uint32_t)(pinfo.size() / V8_PINFO);
    std::vector<uint32_t> wtile;
    std::vector<int32_t> wsegs;
    for (uint32_t t = 0; t < ntile; ++t) {
        for (uint32_t k = 0; k < tiles[t].nseg; k += V8DC_LANES) {
            wtile.push_back(t);
            for (uint32_t l = 0; l < V8DC_LANES; ++l) {
                wsegs.push_back(k + l < tiles[t].nseg ? (int32_t)(tiles[t].seg0 + k + l) : -1);
            }
        }
    }
    const size_t desc = align_up((size_t)nseg * sizeof(tcg_v8_seg) + 16u, 256) +
                        align_up((size_t)ntile * sizeof(tcg_v8_tile) + 16u, 256) + align_up(q.size() * 4u + 16u, 256) +
                        align_up(wtile.size() * 4u + 16u, 256) + align_up(wsegs.size() * 4u + 16u, 256) +
                        align_up(pinfo.size() * 4u + 16u, 256);
    const size_t resb = align_up((size_t)nseg + 16u, 256) + align_up((size_t)ntile + 16u, 256);
    if (!dreserve(C, B_DEC_PKT, pkt_bytes + 256) || !dreserve(C, B_DEC_COEF, nblk * 256u + 256) ||
        !dreserve(C, B_UMAP, (nblk + 31u) / 32u * 4u + 256) ||
        !dreserve(C, B_DEC_TAB, (size_t)ntile * DTAB_BYTES + 256) || !dreserve(C, B_DEC_OUT, out_elems * 2u + 256) ||
        !dreserve(C, B_DEC_RES, resb) || !dreserve(C, B_DESC, desc) || !hreserve(C, 0, desc) || !hreserve(C, 1, resb)) {
        return TCG_ERR_OUT_OF_MEMORY;
    }
    cudaStream_t st = C->stream;
    uint8_t* hd = (uint8_t*)C->h[0].p;
    uint8_t* dd = dptr<uint8_t>(C, B_DESC);
    size_t o = 0;
    auto put = [&](const void* src, size_t n) -> size_t {
        const size_t at = o;
        if (n) { memcpy(hd + o, src, n); }
        o = align_up(o + n, 256);
        return at;
    };
    const size_t o_sg = put(segs.data(), (size_t)nseg * sizeof(tcg_v8_seg));
    const size_t o_tl = put(tiles.data(), (size_t)ntile * sizeof(tcg_v8_tile));
    const size_t o_q = put(q.data(), q.size() * 4u);
    const size_t o_wt = put(wtile.data(), wtile.size() * 4u);
    const size_t o_ws = put(wsegs.data(), wsegs.size() * 4u);
    const size_t o_pi = put(pinfo.data(), pinfo.size() * 4u);
    call_begin(C);
    TCG_CHECK(cudaMemcpyAsync(dd, hd, o, cudaMemcpyHostToDevice, st));
    const tcg_v8_seg* d_sg = (const tcg_v8_seg*)(dd + o_sg);
    const tcg_v8_tile* d_tl = (const tcg_v8_tile*)(dd + o_tl);
    const uint32_t* d_q = (const uint32_t*)(dd + o_q);
    const uint32_t* d_wt = (const uint32_t*)(dd + o_wt);
    const int32_t* d_ws = (const int32_t*)(dd + o_ws);
    const uint32_t* d_pi = (const uint32_t*)(dd + o_pi);
    uint8_t* d_pkt = dptr<uint8_t>(C, B_DEC_PKT);
    for (uint32_t f = 0; f < count; ++f) {
        TCG_CHECK(cudaMemcpyAsync(d_pkt + pkt_off[f], J[f].packet, J[f].size, cudaMemcpyDefault, st));
    }
    int32_t* d_coef = dptr<int32_t>(C, B_DEC_COEF);
    uint8_t* d_tab = dptr<uint8_t>(C, B_DEC_TAB);
    uint16_t* d_out = dptr<uint16_t>(C, B_DEC_OUT);
    uint8_t* d_res = dptr<uint8_t>(C, B_DEC_RES);
    uint8_t* d_fail = d_res;
    uint8_t* d_ok = d_res + align_up((size_t)nseg + 16u, 256);
    TCG_CHECK(cudaMemsetAsync(d_res, 0, resb, st));
    TCG_CHECK(cudaMemsetAsync(d_coef, 0, nblk * 256u, st));
    const DevTables& T = tables();
    if (ntile > 0u) {
        TCG_LAUNCH(C, K_DCRC, k_v8_tcrc, ntile, 256, 0, d_tl, d_pkt, T.crc, d_ok);
        TCG_LAUNCH(C, K_DTABLES, k_v8_dtab, ntile, 32, 0, d_tl, d_pkt, d_tab);
    }
    if (!wtile.empty()) {
        TCG_LAUNCH(C, K_DCHAIN, k_v8_dchain, (uint32_t)wtile.size(), V8DC_LANES, V8D_SMEM, d_sg, d_wt, d_ws, d_pi, d_ok, d_pkt,
                   d_tab, d_coef, d_fail);
    }
    if (nblk > 0u) {
        uint32_t* d_umap = dptr<uint32_t>(C, B_UMAP);
        TCG_LAUNCH(C, K_UNIT_MAP, k_unit_map, (uint32_t)((nblk + 8191u) / 8192u), 256, 0, d_pi, V8_PINFO, nplanes, (uint32_t)nblk,
                   d_umap);
        TCG_LAUNCH(C, K_DIDCT, k_v8_didct, (uint32_t)((nblk + RB_BLOCKS - 1u) / RB_BLOCKS), 256, 0, d_sg, d_pi, nplanes,
                   d_q, d_coef, (uint32_t)nblk, d_umap, d_out);
    }
    for (uint32_t f = 0; f < count; ++f) {
        for (uint32_t p = 0; p < 3u; ++p) {
            const size_t w = J[f].vis_w[p], h = J[f].vis_h[p];
            if (w == 0u || h == 0u) { continue; }
            const size_t pitch = (J[f].dst_stride[p] ? J[f].dst_stride[p] : w) * 2u;
            TCG_CHECK(cudaMemcpy2DAsync(J[f].dst[p], pitch, d_out + out_off[3u * f + p], w * 2u, w * 2u, h,
                                        cudaMemcpyDefault, st));
        }
    }
    uint8_t* hr = (uint8_t*)C->h[1].p;
    TCG_CHECK(cudaMemcpyAsync(hr, d_res, resb, cudaMemcpyDeviceToHost, st));
    TCG_CHECK(cudaGetLastError());
    TCG_CHECK(cudaStreamSynchronize(st));
    call_end(C);
    uint32_t sb0 = 0, tb0 = 0;
    for (uint32_t f = 0; f < count; ++f) {
        memcpy(J[f].seg_fail, hr + sb0, J[f].nseg);
        memcpy(J[f].tile_ok, hr + align_up((size_t)nseg + 16u, 256) + tb0, J[f].ntile);
        sb0 += J[f].nseg;
        tb0 += J[f].ntile;
    }
    return 0;
}

}  // namespace tcg

extern "C" int32_t tcg_decode(const tcg_dec_frame* frames, uint32_t count)
{
    uint32_t first = 0;
    while (first < count && frames[first].skip) { ++first; }
    if (count >= 2u && first < count &&
        (tcg::host_memory(frames[first].packet) || tcg::host_memory(frames[first].dst[0]))) {
        // copy bytes per frame: the packet in, the planes out
        std::vector<uint64_t> bytes(count, 0);
        for (uint32_t f = 0; f < count; ++f) {
            if (frames[f].skip) { continue; }
            bytes[f] = frames[f].size;
            for (uint32_t p = 0; p < frames[f].planes; ++p) { bytes[f] += (uint64_t)frames[f].vis_w[p] * frames[f].vis_h[p] * 2u; }
        }
        uint32_t starts[tcg::PIPE_MAX_CHUNKS + 1];
        const uint32_t k = tcg::pipeline_plan(true, bytes.data(), count, starts);
        if (k > 1u) { return tcg::decode_pipelined(frames, starts, k); }
    }
    tcg::Ctx* c = tcg::ctx_acquire();
    if (c == nullptr) { return TCG_ERR_NOT_IMPLEMENTED; }
    const int32_t rc = tcg::decode_impl(c, frames, count);
    tcg::ctx_release(c);
    return rc;
}

extern "C" int32_t tcg_decode_v8(const tcg_v8_job* jobs, uint32_t count)
{
    if (count == 0u) { return 0; }
    tcg::Ctx* c = tcg::ctx_acquire();
    if (c == nullptr) { return TCG_ERR_NOT_IMPLEMENTED; }
    const int32_t rc = tcg::decode_v8_impl(c, jobs, count);
    tcg::ctx_release(c);
    return rc;
}

extern "C" int32_t tcg_walk_packets(const uint8_t* const* pkts, const size_t* sizes, uint32_t n, uint8_t* host_out)
{
    tcg::Ctx* c = tcg::ctx_acquire();
    if (c == nullptr) { return TCG_ERR_NOT_IMPLEMENTED; }
    const int32_t rc = tcg::walk_impl(c, pkts, sizes, n, host_out);
    tcg::ctx_release(c);
    return rc;
}

extern "C" int32_t tcg_walk_packets_noalloc(const uint8_t* const* pkts, const size_t* sizes, uint32_t n)
{
    if (n == 0u) { return 0; }
    if (n > TCG_NOALLOC_MAX_PACKETS) {
        tcg_host_set_error(TCG_ERR_LIMIT_EXCEEDED, "allocation-free walk: more than 64 packets in one call");
        return TCG_ERR_LIMIT_EXCEEDED;
    }
    int dev = 0;
    TCG_CHECK(cudaGetDevice(&dev));
    // the walk runs on the calling thread's current device: a packet on another
    // device would be read through a peer pointer, so it is refused up front
    for (uint32_t i = 0; i < n; ++i) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, pkts[i]) != cudaSuccess) {
            cudaGetLastError();
            tcg_host_set_error(TCG_ERR_INVALID_ARGUMENT, "allocation-free walk: packet pointer not known to CUDA");
            return TCG_ERR_INVALID_ARGUMENT;
        }
        if (a.type == cudaMemoryTypeDevice && a.device != dev) {
            char msg[160];
            snprintf(msg, sizeof(msg),
                     "allocation-free walk: packet %u is on device %d, the calling thread's current device is %d", i,
                     a.device, dev);
            tcg_host_set_error(TCG_ERR_INVALID_ARGUMENT, msg);
            return TCG_ERR_INVALID_ARGUMENT;
        }
    }
    uint8_t* base = nullptr;
    const int32_t rc = tcg::noalloc_base(dev, &base);
    if (rc != 0) { return rc; }
    uint64_t tab[2u * TCG_NOALLOC_MAX_PACKETS];
    for (uint32_t i = 0; i < n; ++i) {
        tab[i] = (uint64_t)(uintptr_t)pkts[i];
        tab[TCG_NOALLOC_MAX_PACKETS + i] = sizes[i];
    }
    uint8_t* recs = base + 2u * tcg::NA_TABLE;
    TCG_CHECK(cudaMemcpyAsync(base, tab, sizeof(tab), cudaMemcpyHostToDevice, 0));
    // the records of this call start from zero, so nothing an earlier call left is read back
    TCG_CHECK(cudaMemsetAsync(recs, 0, (size_t)n * tcg::WALK_REC, 0));
    tcg::k_walk<<<(n + 63u) / 64u, 64, 0, 0>>>(reinterpret_cast<const uint8_t* const*>(base),
                                                reinterpret_cast<const uint64_t*>(base + tcg::NA_TABLE), n, recs);
    tcg::note_launch(1);
    TCG_CHECK(cudaGetLastError());
    TCG_CHECK(cudaStreamSynchronize(0));
    return 0;
}

extern "C" int32_t tcg_walk_record_noalloc(uint32_t i, uint8_t* host_rec)
{
    if (i >= TCG_NOALLOC_MAX_PACKETS) {
        tcg_host_set_error(TCG_ERR_LIMIT_EXCEEDED, "allocation-free walk: record index beyond 63");
        return TCG_ERR_LIMIT_EXCEEDED;
    }
    int dev = 0;
    TCG_CHECK(cudaGetDevice(&dev));
    uint8_t* base = nullptr;
    const int32_t rc = tcg::noalloc_base(dev, &base);
    if (rc != 0) { return rc; }
    TCG_CHECK(cudaMemcpy(host_rec, base + 2u * tcg::NA_TABLE + (size_t)i * tcg::WALK_REC, tcg::WALK_REC,
                         cudaMemcpyDeviceToHost));
    return 0;
}
