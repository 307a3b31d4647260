// tcg_encode.cu - V7-R2 intra encode on the GPU (any batch of frames).
//
// Pipeline (one stream, no host round trip until the packets are complete):
//   k_fdct      8x8 blocks, 32 per CTA (k_fdct_wide: planes above 12 bits):
//               edge-replicated load, level shift, exact integer forward
//               DCT, dead-zone quantisation -> zigzag coefficients +
//               non-zero mask                       (reference codec.c:1702-1848)
//   k_tokens    DC residuals, run/level categories, per-slice histograms and
//               joint context histograms, op counts  (codec.c:1702-1848, 2116-2151)
//   k_select    per slice: exact double-precision model cost, model choice,
//               row tables, coding tables             (codec.c:2159-2388, rans.c)
//   k_opscan    per slice: reverse exclusive scan of op counts
//   k_opgen     per block: the block's rANS operations in coding order
//   k_chain     one lane per slice: the serial backward rANS state chain
//               with byte renormalisation                (codec.c:2188-2265, 2410-2509)
//   k_alpha     alpha bands: MED residuals + Rice run/level bit packing
//               (codec.c:2969-3010, block_coding.c:456-481)
//   k_pack_*    payload sizes, prefix sums into packet offsets, payload copy,
//               slice CRC-32 + 17-byte headers, frame header size + CRC
//               (codec.c:5203-5225, 5660-5693; frame_header.c:590-631)
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "tcg_common.cuh"
#include "tcg_runtime.h"

namespace tcg {

struct EPlane {
    uint64_t pix_off;    // element offset in the device sample buffer
    uint32_t vis_w, vis_h, coded_w, coded_h, cols, rows;
    uint32_t kind, alpha_shift, bd, q_is_one;
    uint32_t blk0;       // first global colour block
    uint32_t Q[64];
    int64_t fclamp;
    uint32_t seg0;       // V8: first global segment of the plane
    uint32_t sb_log2;    // V8: segment blocks log2 (0 for V7-R2 planes)
    uint32_t Qm[64];     // division by Q[i]: multiplier and shifts (div_magic)
    uint8_t Qsh[64];
};

// Exact division by an invariant divisor (Granlund and Montgomery, "Division
// by invariant integers using multiplication", PLDI 1994, figure 4.1): with
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, every 32-bit n gives
// n / d = (t + ((n - t) >> s1)) >> s2, t = umulhi(m, n), s1 = min(l, 1),
// s2 = max(l - 1, 0). sh packs s1 << 5 | s2.
static void div_magic(uint32_t d, uint32_t* m, uint8_t* sh)
{
    uint32_t l = 0;
    while (l < 32u && (1ull << l) < (uint64_t)d) { ++l; }
    *m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1u);
    *sh = (uint8_t)(l == 0u ? 0u : (1u << 5) | (l - 1u));
}

__device__ __forceinline__ uint32_t div_inv(uint32_t n, uint32_t m, uint32_t sh)
{
    const uint32_t t = __umulhi(m, n);
    return (t + ((n - t) >> (sh >> 5))) >> (sh & 31u);
}

struct ESlice {
    uint32_t frame, plane, kind;
    uint32_t y0, bh, cols;
    uint32_t blk0, nblk;
    uint32_t qdb;
    uint32_t pidx;        // plane index within the frame (slice header field)
    uint64_t op_base;     // u32 units
    uint64_t stage_base;  // bytes
    uint64_t stage_cap;
};

struct ESliceRes {
    uint32_t nops, nbytes, xfin, plen;
    uint32_t payload, crc, err, pad;
    uint64_t pkt_off;     // slice header offset within the frame packet
};

struct EFrame {
    uint32_t slice0, nslices;
    uint64_t pkt_base;
    uint8_t hdr[56];
};

struct EFrameRes {
    uint32_t size, color_payload, alpha_payload, err;
    uint32_t alpha_err, color_slices, alpha_slices, pad;
};

struct EWork {  // token-pass work item: a run of blocks of one colour slice
    uint32_t slice, lb0, n, pad;
};

// ============================== forward DCT ==============================

// Forward transform and quantisation of planes up to 12 bits, 32 blocks per
// CTA of 256 threads: lane b of warp 0 finds block b's plane (from the unit
// map: the plane of the CTA's first block, then a step) and position;
// warp w then loads row w of all 32 blocks (lane = block: a warp reads 512
// contiguous bytes when the blocks lie side by side, edge blocks replicate
// the last column and row), runs the 8-point row pass, and after a barrier
// the column pass of column w with the dead-zone quantisation of its eight
// coefficients (quant.c:310-346; the division by an invariant divisor), which
// land in zigzag order in shared memory; finally each thread stores two
// 16-byte pieces of the CTA's 8 KB of coefficients and 16 lanes OR their
// pieces' non-zero flags into the block's mask. Planes above 12 bits
// (64-bit accumulation and predistortion) go to k_fdct_wide.
constexpr uint32_t FB_BLOCKS = 32u;
constexpr uint32_t FB_P = 65u;  // words per block in shared memory (odd: no bank conflicts)

__global__ void __launch_bounds__(256) k_fdct(const EPlane* __restrict__ planes, const uint32_t* __restrict__ cplanes,
                                              uint32_t ncp, uint32_t total, const uint16_t* __restrict__ pix,
                                              int32_t* __restrict__ coef, uint64_t* __restrict__ mask,
                                              const uint32_t* __restrict__ pstart, const uint32_t* __restrict__ umap)
{
    __shared__ int32_t sa[FB_BLOCKS * FB_P];   // row-pass output, natural order
    __shared__ int32_t sq[FB_BLOCKS * FB_P];   // quantised, zigzag order
    __shared__ uint32_t s_pl[FB_BLOCKS], s_bx[FB_BLOCKS], s_by[FB_BLOCKS];
    __shared__ uint8_t s_zinv[64];
    const uint32_t t = threadIdx.x, w = t >> 5, lane = t & 31u;
    const uint32_t gb0 = blockIdx.x * FB_BLOCKS;
    if (t < 64u) { s_zinv[k_zigzag[t]] = (uint8_t)t; }
    if (t < FB_BLOCKS) {
        const uint32_t gb = gb0 + t;
        uint32_t pl = 0xFFFFFFFFu, bx = 0, by = 0;
        if (gb < total) {
            const uint32_t lo = unit_of(pstart, 1u, ncp, umap[blockIdx.x], gb);
            const EPlane& P = planes[cplanes[lo]];
            if (P.bd <= 12u) {
                pl = cplanes[lo];
                const uint32_t lb = gb - P.blk0;
                bx = lb % P.cols;
                by = lb / P.cols;
            }
        }
        s_pl[t] = pl; s_bx[t] = bx; s_by[t] = by;
    }
    __syncthreads();
    const uint32_t b = lane;
    const uint32_t pl = s_pl[b];
    if (pl != 0xFFFFFFFFu) {  // row pass: row y = w
        const EPlane& P = planes[pl];
        const uint32_t bx = s_bx[b], by = s_by[b], y = w;
        const uint32_t sy = min(by * 8u + y, P.vis_h - 1u);
        const uint16_t* row = pix + P.pix_off + (size_t)sy * P.vis_w;
        const int32_t mid = 1 << (P.bd - 1u);
        uint32_t u[8];
        // planes start on 64-sample boundaries: an inner block of a plane whose
        // width is a multiple of 8 reads its row with one 16-byte load
        if ((P.vis_w & 7u) == 0u && bx * 8u + 8u <= P.vis_w) {
            const uint4 r = __ldg(reinterpret_cast<const uint4*>(row + bx * 8u));
            u[0] = r.x & 0xFFFFu; u[1] = r.x >> 16; u[2] = r.y & 0xFFFFu; u[3] = r.y >> 16;
            u[4] = r.z & 0xFFFFu; u[5] = r.z >> 16; u[6] = r.w & 0xFFFFu; u[7] = r.w >> 16;
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) { u[k] = __ldg(row + min(bx * 8u + (uint32_t)k, P.vis_w - 1u)); }
        }
        int32_t x[8], A[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) { x[k] = (int32_t)(int16_t)((int32_t)u[k] - mid); }
        fwd8<int32_t>(x, A);
#pragma unroll
        for (int v = 0; v < 8; ++v) { sa[b * FB_P + y * 8u + v] = A[v]; }
    }
    __syncthreads();
    if (pl != 0xFFFFFFFFu) {  // column pass and quantisation: column v = w
        const EPlane& P = planes[pl];
        const uint32_t v = w;
        int32_t col[8], F[8];
#pragma unroll
        for (int y = 0; y < 8; ++y) { col[y] = sa[b * FB_P + y * 8u + v]; }
        fwd8<int32_t>(col, F);
        const int32_t fc = (int32_t)P.fclamp;  // 2^25 up to 12 bits
        const bool one = P.q_is_one != 0u;
#pragma unroll
        for (int uu = 0; uu < 8; ++uu) {
            const uint32_t i = (uint32_t)uu * 8u + v;  // natural position
            const int32_t c = min(max(F[uu], -fc), fc);
            const uint32_t mag = (uint32_t)abs(c);
            uint32_t qm;
            if (one) {
                qm = mag;
            } else {
                const uint32_t Q = P.Q[i];
                const uint32_t dz = i == 0u ? 0u : Q >> 2;
                const uint32_t num = mag + (Q >> 1);
                qm = num > dz ? div_inv(num - dz, P.Qm[i], P.Qsh[i]) : 0u;
            }
            sq[b * FB_P + s_zinv[i]] = c < 0 ? -(int32_t)qm : (int32_t)qm;
        }
    }
    __syncthreads();
    // coefficients out, zigzag order, and the non-zero masks
#pragma unroll
    for (uint32_t h = 0; h < 2u; ++h) {
        const uint32_t idx = t + 256u * h;  // 16-byte piece of the CTA's coefficients
        const uint32_t bb = idx >> 4, i0 = (idx & 15u) * 4u;
        const bool live = s_pl[bb] != 0xFFFFFFFFu;
        uint32_t m = 0;
        if (live) {
            int4 q;
            q.x = sq[bb * FB_P + i0]; q.y = sq[bb * FB_P + i0 + 1u];
            q.z = sq[bb * FB_P + i0 + 2u]; q.w = sq[bb * FB_P + i0 + 3u];
            reinterpret_cast<int4*>(coef + (size_t)gb0 * 64u)[idx] = q;
            m = (uint32_t)((q.x != 0) | ((q.y != 0) << 1) | ((q.z != 0) << 2) | ((q.w != 0) << 3)) << (i0 & 31u);
        }
        // the block's 16 pieces sit in 16 neighbouring lanes: the first 8 hold
        // positions 0..31, the next 8 positions 32..63
#pragma unroll
        for (uint32_t d = 1; d < 8u; d <<= 1) { m |= __shfl_xor_sync(0xFFFFFFFFu, m, d); }
        const uint32_t hi = __shfl_down_sync(0xFFFFFFFFu, m, 8);
        if (live && (idx & 15u) == 0u) { mask[gb0 + bb] = ((uint64_t)hi << 32 | m) & ~(uint64_t)1; }
    }
}

__global__ void __launch_bounds__(128) k_fdct_wide(const EPlane* __restrict__ planes, const uint32_t* __restrict__ cplanes,
                                              uint32_t ncp, uint32_t total, const uint16_t* __restrict__ pix,
                                              int32_t* __restrict__ coef, uint64_t* __restrict__ mask)
{
    const uint32_t gb = blockIdx.x * blockDim.x + threadIdx.x;
    if (gb >= total) { return; }
    int lo = 0, hi = (int)ncp - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (planes[cplanes[mid]].blk0 <= gb) { lo = mid; } else { hi = mid - 1; }
    }
    const EPlane& P = planes[cplanes[lo]];
    if (P.bd <= 12u) { return; }  // k_fdct's blocks
    const uint32_t lb = gb - P.blk0;
    const uint32_t bx = lb % P.cols, by = lb / P.cols;
    const uint16_t* src = pix + P.pix_off;
    const int32_t mid = 1 << (P.bd - 1u);
    const bool wide = true;
    int32_t x[64], F[64];
    // a block inside the visible plane with 16-byte aligned rows (planes start
    // on 64-sample boundaries) reads each row with one load; edge blocks
    // replicate the last column and row
    const bool inner = (P.vis_w & 7u) == 0u && bx * 8u + 8u <= P.vis_w && by * 8u + 8u <= P.vis_h;
#pragma unroll
    for (int y = 0; y < 8; ++y) {
        const uint32_t sy = min(by * 8u + (uint32_t)y, P.vis_h - 1u);
        const uint16_t* row = src + (size_t)sy * P.vis_w;
        uint32_t u[8];
        if (inner) {
            const uint4 r = __ldg(reinterpret_cast<const uint4*>(row + bx * 8u));
            u[0] = r.x & 0xFFFFu; u[1] = r.x >> 16; u[2] = r.y & 0xFFFFu; u[3] = r.y >> 16;
            u[4] = r.z & 0xFFFFu; u[5] = r.z >> 16; u[6] = r.w & 0xFFFFu; u[7] = r.w >> 16;
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) { u[k] = __ldg(row + min(bx * 8u + (uint32_t)k, P.vis_w - 1u)); }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int32_t d = (int32_t)u[k] - mid;
            x[y * 8 + k] = wide ? d : (int32_t)(int16_t)d;
        }
    }
    fdct8x8_wide(x, F);
    // dead-zone quantisation (quant.c:310-346): q = sign*((|F|+Q/2-dz)/Q), dz = Q/4 (AC)
    int32_t q[64];
    const int64_t fc = P.fclamp;
#pragma unroll
    for (int i = 0; i < 64; ++i) {
        int64_t v = F[i];
        v = v > fc ? fc : (v < -fc ? -fc : v);
        const uint32_t mag = (uint32_t)(v < 0 ? -v : v);
        uint32_t qm;
        if (P.q_is_one) {
            qm = mag;
        } else {
            const uint32_t Q = P.Q[i];
            const uint32_t dz = i == 0 ? 0u : Q >> 2;
            const uint32_t num = mag + (Q >> 1);
            qm = num > dz ? (num - dz) / Q : 0u;
        }
        q[i] = v < 0 ? -(int32_t)qm : (int32_t)qm;
    }
    uint64_t m = 0;
    int4* out = reinterpret_cast<int4*>(coef + (size_t)gb * 64u);
#pragma unroll
    for (int p = 0; p < 64; p += 4) {
        int4 v;
        v.x = q[k_zigzag[p]]; v.y = q[k_zigzag[p + 1]]; v.z = q[k_zigzag[p + 2]]; v.w = q[k_zigzag[p + 3]];
        m |= (uint64_t)(v.x != 0) << p | (uint64_t)(v.y != 0) << (p + 1) | (uint64_t)(v.z != 0) << (p + 2) |
             (uint64_t)(v.w != 0) << (p + 3);
        out[p >> 2] = v;
    }
    mask[gb] = m & ~(uint64_t)1;
}

// ======================= tokens + histograms + op counts =======================

__device__ __forceinline__ uint32_t block_dcm(const int32_t* coef, uint32_t gb, uint32_t lb, uint32_t cols, bool* viol)
{
    const uint32_t bx = lb % cols, by = lb / cols;
    const int32_t q0 = coef[(size_t)gb * 64u];
    const int32_t l = bx > 0u ? coef[(size_t)(gb - 1u) * 64u] : 0;
    const int32_t t = by > 0u ? coef[(size_t)(gb - cols) * 64u] : 0;
    uint32_t dcm = map_s(q0 - dc_pred(bx > 0u, l, by > 0u, t));
    if (dcm > 0x0FFFFFFFu) { dcm = 0x0FFFFFFFu; *viol = true; }
    return dcm;
}

__global__ void __launch_bounds__(256) k_tokens(const EWork* __restrict__ work, const ESlice* __restrict__ slices,
                                                const int32_t* __restrict__ coef, const uint64_t* __restrict__ mask,
                                                uint32_t* __restrict__ dcm_out, uint32_t* __restrict__ nops_out,
                                                uint32_t* __restrict__ hist, ESliceRes* __restrict__ sres)
{
    extern __shared__ uint32_t sh[];  // [H_BINS][32] lane-replicated counters
    const EWork w = work[blockIdx.x];
    const ESlice& S = slices[w.slice];
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t i = threadIdx.x; i < H_BINS * 32u; i += blockDim.x) { sh[i] = 0u; }
    __syncthreads();
    bool viol = false;
    if (threadIdx.x < w.n) {
        const uint32_t lb = w.lb0 + threadIdx.x;
        const uint32_t gb = S.blk0 + lb;
        const uint32_t dcm = block_dcm(coef, gb, lb, S.cols, &viol);
        const uint32_t dcc = bitlen32(dcm);
        uint32_t ctx = 0u;
        if (lb > 0u) {
            bool dummy = false;
            ctx = dcp_ctx(bitlen32(block_dcm(coef, gb - 1u, lb - 1u, S.cols, &dummy)), true);
        }
        atomicAdd(&sh[(H_DC + dcc) * 32u + lane], 1u);
        atomicAdd(&sh[(H_JDC + ctx * DC_SYMS + dcc) * 32u + lane], 1u);
        uint32_t nops = 2u + suffix_chunks(dcc);  // EOB + DC symbol + DC suffix
        const uint64_t m = mask[gb];
        uint32_t prev = 0u, pcat = 0u;
        bool has = false;
        // the whole block (zigzag order) in 16 independent loads, then the
        // positions in order over registers
        int32_t cv[64];
        const int4* c4 = reinterpret_cast<const int4*>(coef + (size_t)gb * 64u);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int4 v = c4[i];
            cv[4 * i] = v.x; cv[4 * i + 1] = v.y; cv[4 * i + 2] = v.z; cv[4 * i + 3] = v.w;
        }
#pragma unroll
        for (uint32_t p = 1; p < 64u; ++p) {
            if (((m >> p) & 1u) == 0u) { continue; }
            uint32_t lm = map_s(cv[p]);
            if (lm > 0x07FFFFFFu) { lm = 0x07FFFFFFu; viol = true; }
            const uint32_t cat = bitlen32(lm);
            const uint32_t run = p - prev - 1u;
            atomicAdd(&sh[(H_RUN + run) * 32u + lane], 1u);
            atomicAdd(&sh[(H_LVL + cat) * 32u + lane], 1u);
            atomicAdd(&sh[(H_JPOS + pos_ctx(p) * LVL_SYMS + cat) * 32u + lane], 1u);
            atomicAdd(&sh[(H_JPREV + prev_ctx(pcat, has) * LVL_SYMS + cat) * 32u + lane], 1u);
            nops += 2u + suffix_chunks(cat);
            prev = p;
            pcat = cat;
            has = true;
        }
        atomicAdd(&sh[(H_RUN + 63u) * 32u + lane], 1u);
        dcm_out[gb] = dcm;
        nops_out[gb] = nops;
    }
    if (__syncthreads_or(viol) && threadIdx.x == 0) { atomicOr(&sres[w.slice].err, 1u); }
    uint32_t* g = hist + (size_t)w.slice * H_BINS;
    for (uint32_t b = threadIdx.x; b < H_BINS; b += blockDim.x) {
        uint32_t s = 0;
#pragma unroll 8
        for (uint32_t r = 0; r < 32u; ++r) { s += sh[b * 32u + ((r + b) & 31u)]; }
        if (s != 0u) { atomicAdd(&g[b], s); }
    }
}

// ============================ per-slice model choice ============================

// One 32-thread block per colour slice. Row models are normalised in parallel
// (one row per lane); the five candidate costs are then accumulated each by a
// single lane in the reference order with separately rounded double ops.
__global__ void __launch_bounds__(32) k_select(const ESlice* __restrict__ slices, const uint32_t* __restrict__ cslices,
                                               const uint32_t* __restrict__ hist, const double* __restrict__ log2t,
                                               uint32_t* __restrict__ stab, uint8_t* __restrict__ prefix,
                                               ESliceRes* __restrict__ sres)
{
    __shared__ uint32_t h[H_BINS];
    __shared__ uint8_t rb[17][64];
    __shared__ uint16_t rf[17][64];
    __shared__ uint16_t rc[17][64];
    __shared__ double cost[5];
    __shared__ uint32_t sel[2];
    const uint32_t si = cslices[blockIdx.x];
    const uint32_t t = threadIdx.x;
    for (uint32_t i = t; i < H_BINS; i += 32u) { h[i] = hist[(size_t)si * H_BINS + i]; }
    __syncwarp();
    // rows: 0 lvl, 1-4 jpos, 5-9 jprev, 10 dc, 11-15 jdc, 16 run
    if (t < 17u) {
        const uint32_t* cnt;
        uint32_t n;
        if (t == 0u) { cnt = h + H_LVL; n = LVL_SYMS; }
        else if (t <= 4u) { cnt = h + H_JPOS + (t - 1u) * LVL_SYMS; n = LVL_SYMS; }
        else if (t <= 9u) { cnt = h + H_JPREV + (t - 5u) * LVL_SYMS; n = LVL_SYMS; }
        else if (t == 10u) { cnt = h + H_DC; n = DC_SYMS; }
        else if (t <= 15u) { cnt = h + H_JDC + (t - 11u) * DC_SYMS; n = DC_SYMS; }
        else { cnt = h + H_RUN; n = RUN_SYMS; }
        row_encode(rb[t], n, cnt);
        model_from_bytes(rb[t], n, rf[t], rc[t]);
    }
    __syncwarp();
    if (t < 5u) {
        uint32_t r0, nr, n, base, stride;
        double extra;
        if (t == 0u) { r0 = 0; nr = 1; n = LVL_SYMS; base = H_LVL; stride = LVL_SYMS; extra = 8.0 * 28.0; }
        else if (t == 1u) { r0 = 1; nr = 4; n = LVL_SYMS; base = H_JPOS; stride = LVL_SYMS; extra = 8.0 * 112.0; }
        else if (t == 2u) { r0 = 5; nr = 5; n = LVL_SYMS; base = H_JPREV; stride = LVL_SYMS; extra = 8.0 * 140.0; }
        else if (t == 3u) { r0 = 10; nr = 1; n = DC_SYMS; base = H_DC; stride = DC_SYMS; extra = 8.0 * 29.0; }
        else { r0 = 11; nr = 5; n = DC_SYMS; base = H_JDC; stride = DC_SYMS; extra = 8.0 * 145.0; }
        double bits = 0.0;
        for (uint32_t r = 0; r < nr; ++r) {
            for (uint32_t s = 0; s < n; ++s) {
                const uint32_t c = h[base + r * stride + s];
                if (c != 0u) {
                    bits = __dadd_rn(bits, __dmul_rn((double)c, __dsub_rn(12.0, log2t[rf[r0 + r][s]])));
                }
            }
        }
        cost[t] = __dadd_rn(bits, extra);
    }
    __syncwarp();
    if (t == 0u) {
        uint32_t lm = 0;
        double best = cost[0];
        if (cost[1] < best) { best = cost[1]; lm = 1; }
        if (cost[2] < best) { lm = 2; }
        sel[0] = lm;
        sel[1] = cost[4] < cost[3] ? 1u : 0u;
    }
    __syncwarp();
    const uint32_t lm = sel[0], dm = sel[1];
    const uint32_t nd = dm ? DCP_CTX : 1u, nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u;
    const uint32_t dr0 = dm ? 11u : 10u, lr0 = lm == 1u ? 1u : lm == 2u ? 5u : 0u;
    uint8_t* pre = prefix + (size_t)si * PREFIX_MAX;
    const uint32_t plen = 1u + nd * DC_SYMS + RUN_SYMS + nl * LVL_SYMS;
    for (uint32_t i = t; i < plen; i += 32u) {
        uint8_t v;
        if (i == 0u) { v = (uint8_t)(lm | (dm << 2)); }
        else if (i < 1u + nd * DC_SYMS) { const uint32_t j = i - 1u; v = rb[dr0 + j / DC_SYMS][j % DC_SYMS]; }
        else if (i < 1u + nd * DC_SYMS + RUN_SYMS) { v = rb[16][i - 1u - nd * DC_SYMS]; }
        else { const uint32_t j = i - 1u - nd * DC_SYMS - RUN_SYMS; v = rb[lr0 + j / LVL_SYMS][j % LVL_SYMS]; }
        pre[i] = v;
    }
    uint32_t* tb = stab + (size_t)si * T_SIZE;
    for (uint32_t i = t; i < T_SIZE; i += 32u) {
        uint32_t r, s;
        if (i < T_RUN) { r = dr0 + (i / DC_SYMS < nd ? i / DC_SYMS : 0u); s = i % DC_SYMS; }
        else if (i < T_LVL) { r = 16u; s = i - T_RUN; }
        else { const uint32_t j = i - T_LVL; r = lr0 + (j / LVL_SYMS < nl ? j / LVL_SYMS : 0u); s = j % LVL_SYMS; }
        tb[i] = ((uint32_t)rf[r][s] << 12) | rc[r][s];
    }
    if (t == 0u) { sres[si].plen = plen | (lm << 16) | (dm << 20); }
}

// ======================= op counts -> offsets (reverse scan) =======================

__global__ void __launch_bounds__(1024) k_opscan(const ESlice* __restrict__ slices, const uint32_t* __restrict__ cslices,
                                                 const uint32_t* __restrict__ nops, uint32_t* __restrict__ opoff,
                                                 uint32_t* __restrict__ ops, ESliceRes* __restrict__ sres)
{
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    const uint32_t si = cslices[blockIdx.x];
    const ESlice& S = slices[si];
    const uint32_t n = S.nblk;
    if (threadIdx.x == 0) { carry = 0u; }
    __syncthreads();
    // position r counts blocks from the end of the slice (coding order)
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t r = base + threadIdx.x;
        const uint32_t v = r < n ? nops[S.blk0 + (n - 1u - r)] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
            if ((threadIdx.x & 31u) >= (uint32_t)d) { x += y; }
        }
        if ((threadIdx.x & 31u) == 31u) { wsum[threadIdx.x >> 5] = x; }
        __syncthreads();
        if (threadIdx.x < 32u) {
            uint32_t s = threadIdx.x < (blockDim.x >> 5) ? wsum[threadIdx.x] : 0u;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, d);
                if (threadIdx.x >= (uint32_t)d) { s += y; }
            }
            wsum[threadIdx.x] = s;
        }
        __syncthreads();
        const uint32_t wpre = (threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1u] : 0u;
        if (r < n) { opoff[S.blk0 + (n - 1u - r)] = carry + wpre + x - v; }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1u) { carry += wpre + x; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { sres[si].nops = carry; }
    // identity operations (word 0) from the count up to the next multiple of
    // 32, so the chain reads whole 32-operation iterations without masking
    // (a slice window holds 256 words past its largest count)
    if (threadIdx.x < 32u && carry + threadIdx.x < ((carry + 31u) & ~31u)) {
        ops[S.op_base + carry + threadIdx.x] = 0u;
    }
}

// ============================== op generation ==============================
// op word: bits 23..31 index into the slice's coding table, bits 0..22 a raw
// value. Index 0..23 is a raw chunk of that many bits (0 = identity); index
// 24 + t is the symbol whose frequency/cumulative word sits at t in the
// slice's symbol table (T_DC / T_RUN / T_LVL layout).

constexpr uint32_t OP_CHUNKS = 24u;
constexpr uint32_t OP_ENTRIES = OP_CHUNKS + T_SIZE;

__device__ __forceinline__ uint32_t op_chunk(uint32_t w, uint32_t v) { return (w << 23) | (v & ((1u << w) - 1u)); }
__device__ __forceinline__ uint32_t op_sym(uint32_t t) { return (OP_CHUNKS + t) << 23; }

__device__ __forceinline__ void put_suffix_ops(uint32_t*& o, uint32_t cat, uint32_t m)
{
    if (cat <= 1u) { return; }
    uint32_t b = cat - 1u;
    if (b > 23u) { *o++ = op_chunk(b - 16u, m >> 16); b = 16u; }
    *o++ = op_chunk(b, m);
}

// One warp per 8x8 block: lane j owns zigzag positions j and j+32. The block's
// operations are, in coding order, the end-of-block run, then for every
// non-zero AC position from the highest down its suffix chunk(s), level and
// run, then the DC suffix and DC category; a warp suffix-sum over positions
// gives each lane the offset of its positions' operations, so the block's
// words are written by neighbouring lanes.
__global__ void __launch_bounds__(256) k_opgen(const EWork* __restrict__ work, const ESlice* __restrict__ slices,
                                               const int32_t* __restrict__ coef, const uint64_t* __restrict__ mask,
                                               const uint32_t* __restrict__ dcm, const uint32_t* __restrict__ opoff,
                                               const ESliceRes* __restrict__ sres, uint32_t* __restrict__ ops)
{
    __shared__ uint8_t cats[8][64];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const EWork w = work[blockIdx.x];
    const uint32_t k = blockIdx.y * 8u + warp;
    if (k >= w.n) { return; }  // whole warp
    const ESlice& S = slices[w.slice];
    const uint32_t lb = w.lb0 + k;
    const uint32_t gb = S.blk0 + lb;
    const uint32_t pl = sres[w.slice].plen;
    const uint32_t lmod = (pl >> 16) & 3u, dmod = (pl >> 20) & 1u;
    uint32_t* o = ops + S.op_base + opoff[gb];
    const int32_t* c = coef + (size_t)gb * 64u;
    const uint64_t m = mask[gb];  // AC positions only (bit 0 clear)
    uint32_t lmv[2], cat[2], cnt[2];
#pragma unroll
    for (uint32_t h = 0; h < 2u; ++h) {
        const uint32_t p = lane + 32u * h;
        const bool nz = ((m >> p) & 1u) != 0u;
        const uint32_t lv = nz ? map_s(c[p]) : 0u;
        lmv[h] = lv > 0x07FFFFFFu ? 0x07FFFFFFu : lv;
        cat[h] = nz ? bitlen32(lmv[h]) : 0u;
        cnt[h] = nz ? 2u + suffix_chunks(cat[h]) : 0u;
        cats[warp][p] = (uint8_t)cat[h];
    }
    // operations of the positions above each of this lane's two positions
    const uint32_t packed = cnt[0] | (cnt[1] << 16);
    uint32_t incl = packed;
#pragma unroll
    for (uint32_t d = 1; d < 32u; d <<= 1) {
        const uint32_t t = __shfl_down_sync(0xFFFFFFFFu, incl, d);
        if (lane + d < 32u) { incl += t; }
    }
    const uint32_t above = incl - packed;
    const uint32_t all = __shfl_sync(0xFFFFFFFFu, incl, 0);
    const uint32_t hi_total = all >> 16, total = (all & 0xFFFFu) + hi_total;
    __syncwarp();
#pragma unroll
    for (uint32_t h = 0; h < 2u; ++h) {
        if (cnt[h] == 0u) { continue; }
        const uint32_t p = lane + 32u * h;
        uint32_t* q = o + 1u + (h ? (above >> 16) : hi_total + (above & 0xFFFFu));
        const uint64_t lower = m & ((1ull << p) - 1ull);
        const uint32_t below = lower != 0u ? 63u - (uint32_t)__clzll((long long)lower) : 0u;
        put_suffix_ops(q, cat[h], lmv[h]);
        uint32_t ctx = 0u;
        if (lmod == 1u) {
            ctx = pos_ctx(p);
        } else if (lmod == 2u) {
            ctx = prev_ctx(lower != 0u ? cats[warp][below] : 0u, lower != 0u);
        }
        *q++ = op_sym(T_LVL + ctx * LVL_SYMS + cat[h]);
        *q = op_sym(T_RUN + (p - below - 1u));
    }
    if (lane == 0u) {
        o[0] = op_sym(T_RUN + 63u);  // EOB
        uint32_t* q = o + 1u + total;
        const uint32_t dm = dcm[gb];
        const uint32_t ds = bitlen32(dm);
        put_suffix_ops(q, ds, dm);
        const uint32_t dctx = dmod ? dcp_ctx(lb > 0u ? bitlen32(dcm[gb - 1u]) : 0u, lb > 0u) : 0u;
        *q = op_sym(T_DC + dctx * DC_SYMS + ds);
    }
}

// =============================== rANS chains ===============================

// Coding-table entry of one operation: renormalisation threshold, division
// magic m and shift l (q = umulhi(2x, m) >> l = x / f for x < 2^31), additive
// term, and B << 5 | l (a shift takes its amount from the low 5 bits, so l
// needs no extraction). Every operation is then
//   x <- q * B + x + add  after renormalisation against lim:
// a symbol of frequency f has B = 4096 - f, add = cum (x/f*4096 + x%f + cum);
// a raw chunk of w bits has f = 1 (q = x), B = 2^w - 1, add = the value
// (x * 2^w + value); the 0-bit chunk is the identity.
__device__ __forceinline__ uint4 chunk_entry(uint32_t w)
{
    return make_uint4(1u << (31u - w), 0x80000000u, 0u, ((1u << w) - 1u) << 5);
}

__device__ __forceinline__ uint4 symbol_entry(uint32_t word, const uint32_t* __restrict__ div_m,
                                              const uint8_t* __restrict__ div_l)
{
    const uint32_t f = word >> 12;
    if (f == 0u) { return chunk_entry(0u); }  // symbol absent from the model: never coded
    return make_uint4(f << 19, __ldg(div_m + f), word & 0xFFFu, ((4096u - f) << 5) | (uint32_t)__ldg(div_l + f));
}

// One coding operation, branch-free; emitted bytes (0..3, least significant
// first) are stored downwards from p.
__device__ __forceinline__ void enc_step(uint32_t& x, uint8_t*& p, uint32_t o, const uint4* __restrict__ tab)
{
    const uint4 e = tab[o >> 23];
    const uint32_t v = o & 0x7FFFFFu;
    const uint32_t x8 = x >> 8, x16 = x >> 16, x24 = x >> 24;
    const bool c1 = x >= e.x, c2 = x8 >= e.x, c3 = x16 >= e.x;
    const uint32_t xr = c2 ? (c3 ? x24 : x16) : (c1 ? x8 : x);
    const uint32_t q = __funnelshift_r(__umulhi(xr << 1, e.y), 0u, e.w);  // >> l (e.w & 31)
    const uint32_t xn = q * (e.w >> 5) + (xr + e.z + v);
    if (c1) { p[-1] = (uint8_t)x; }
    if (c2) { p[-2] = (uint8_t)x8; }
    if (c3) { p[-3] = (uint8_t)x16; }
    p -= c2 ? (c3 ? 3 : 2) : (c1 ? 1 : 0);
    x = xn;
}

// Four consecutive operations of a slice or segment (group g). Its window
// holds identity operations from its count to the next multiple of the
// chain's iteration (32 operations for k_chain, 64 for k_v8_chain), and
// every group a chain loads lies within the window (at most 127 words past
// the count; a window has 256 words to spare).
__device__ __forceinline__ uint4 op_group(const uint4* __restrict__ op4, uint32_t g, uint32_t)
{
    return __ldg(op4 + g);
}

#define ENC_GROUP(v)                  \
    do {                              \
        enc_step(x, p, (v).x, tab);   \
        enc_step(x, p, (v).y, tab);   \
        enc_step(x, p, (v).z, tab);   \
        enc_step(x, p, (v).w, tab);   \
    } while (0)

constexpr uint32_t CHAIN_LANES = 32u;
constexpr size_t CHAIN_SMEM = (size_t)CHAIN_LANES * OP_ENTRIES * sizeof(uint4);

// One lane per colour slice. The lane expands its slice's symbol table into
// per-operation coding entries in shared memory, then walks the operations in
// coding order, 32 per iteration with the operation words loaded 32 ahead of
// their use. Bytes go downwards from the end of the lane's staging
// window, so the stream reads forwards.
__global__ void __launch_bounds__(CHAIN_LANES) k_chain(const ESlice* __restrict__ slices,
                                                       const uint32_t* __restrict__ order, uint32_t n,
                                                       const uint32_t* __restrict__ ops,
                                                       const uint32_t* __restrict__ stab,
                                                       const uint32_t* __restrict__ div_m,
                                                       const uint8_t* __restrict__ div_l, uint8_t* __restrict__ stage,
                                                       ESliceRes* __restrict__ sres)
{
    extern __shared__ uint4 chain_tab[];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) { return; }
    const uint32_t si = order[i];
    uint4* tab = chain_tab + (size_t)threadIdx.x * OP_ENTRIES;
    for (uint32_t w = 0; w < OP_CHUNKS; ++w) { tab[w] = chunk_entry(w); }
    const uint32_t* st = stab + (size_t)si * T_SIZE;
    for (uint32_t t = 0; t < T_SIZE; ++t) { tab[OP_CHUNKS + t] = symbol_entry(__ldg(st + t), div_m, div_l); }
    const ESlice& S = slices[si];
    const uint32_t nops = sres[si].nops;
    // op windows start on 1 KiB boundaries (256 words per block) and hold whole groups
    const uint4* op4 = reinterpret_cast<const uint4*>(ops + S.op_base);
    uint8_t* const end = stage + S.stage_base + S.stage_cap;  // emitted byte k lives at end[-1-k]
    uint8_t* p = end;
    uint32_t x = RANS_L;
    // eight groups (32 operations) in registers, each reloaded eight groups ahead
    // of its use, and an L1 prefetch 512 bytes ahead
    uint4 q0 = op_group(op4, 0u, nops), q1 = op_group(op4, 1u, nops);
    uint4 q2 = op_group(op4, 2u, nops), q3 = op_group(op4, 3u, nops);
    uint4 q4 = op_group(op4, 4u, nops), q5 = op_group(op4, 5u, nops);
    uint4 q6 = op_group(op4, 6u, nops), q7 = op_group(op4, 7u, nops);
    for (uint32_t g = 0; 4u * g < nops; g += 8u) {
        const uint32_t pf = (uint32_t)(4u * (g + 32u) < nops);
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, 0;\n\t@p prefetch.global.L1 [%0];\n\t}"
                     :: "l"(op4 + g + 32u), "r"(pf));
        ENC_GROUP(q0); q0 = op_group(op4, g + 8u, nops);
        ENC_GROUP(q1); q1 = op_group(op4, g + 9u, nops);
        ENC_GROUP(q2); q2 = op_group(op4, g + 10u, nops);
        ENC_GROUP(q3); q3 = op_group(op4, g + 11u, nops);
        ENC_GROUP(q4); q4 = op_group(op4, g + 12u, nops);
        ENC_GROUP(q5); q5 = op_group(op4, g + 13u, nops);
        ENC_GROUP(q6); q6 = op_group(op4, g + 14u, nops);
        ENC_GROUP(q7); q7 = op_group(op4, g + 15u, nops);
    }
    sres[si].nbytes = (uint32_t)(end - p);
    sres[si].xfin = x;
}

// ================================ alpha bands ================================

__device__ __forceinline__ uint32_t rice_len(uint32_t k, uint32_t m)
{
    const uint32_t q = m >> k;
    return q <= 30u ? q + 1u + k : 63u;
}

// OR an n-bit field (n <= 32, MSB first) into a zeroed byte stream at bit o.
__device__ __forceinline__ void put_bits_or(uint8_t* base, uint64_t o, uint32_t n, uint32_t v)
{
    while (n > 0u) {
        const uint32_t room = 8u - (uint32_t)(o & 7u);
        const uint32_t take = n < room ? n : room;
        const uint32_t piece = (v >> (n - take)) & ((1u << take) - 1u);
        const uint8_t b = (uint8_t)(piece << (room - take));
        uint8_t* p = base + (o >> 3);
        uint32_t* wd = reinterpret_cast<uint32_t*>((uintptr_t)p & ~(uintptr_t)3);
        atomicOr(wd, (uint32_t)b << (8u * ((uintptr_t)p & 3u)));
        o += take;
        n -= take;
    }
}

__device__ __forceinline__ void put_rice(uint8_t* base, uint64_t o, uint32_t k, uint32_t m)
{
    const uint32_t q = m >> k;
    if (q <= 30u) {
        const uint32_t ones = q == 0u ? 0u : (0xFFFFFFFFu >> (32u - q));
        put_bits_or(base, o, q + 1u, ones << 1);  // q ones then a zero
        if (k > 0u) { put_bits_or(base, o + q + 1u, k, m & ((1u << k) - 1u)); }
    } else {
        put_bits_or(base, o, 31u, 0x7FFFFFFFu);
        put_bits_or(base, o + 31u, 32u, m);
    }
}

__device__ __forceinline__ uint32_t alpha_sample(const uint16_t* src, const EPlane& P, uint32_t x, uint32_t y)
{
    const uint32_t sx = min(x, P.vis_w - 1u), sy = min(y, P.vis_h - 1u);
    uint32_t v = __ldg(src + (size_t)sy * P.vis_w + sx);
    if (P.alpha_shift != 0u) {
        const uint32_t s = P.alpha_shift, top = (0xFFFFu >> s) << s;
        v = ((v + (1u << (s - 1u))) >> s) << s;
        v = v > top ? top : v;
    }
    return v;
}

__device__ __forceinline__ int32_t alpha_residual(const uint16_t* src, const EPlane& P, uint32_t py0, uint32_t idx)
{
    const uint32_t w = P.coded_w;
    const uint32_t y = idx / w, x = idx % w;
    const int32_t a = (int32_t)alpha_sample(src, P, x, py0 + y);
    int32_t pred;
    if (y == 0u) {
        pred = x == 0u ? 0 : (int32_t)alpha_sample(src, P, x - 1u, py0);
    } else if (x == 0u) {
        pred = (int32_t)alpha_sample(src, P, 0u, py0 + y - 1u);
    } else {
        const int32_t l = (int32_t)alpha_sample(src, P, x - 1u, py0 + y);
        const int32_t u = (int32_t)alpha_sample(src, P, x, py0 + y - 1u);
        const int32_t ul = (int32_t)alpha_sample(src, P, x - 1u, py0 + y - 1u);
        if (ul >= l && ul >= u) { pred = l < u ? l : u; }
        else if (ul <= l && ul <= u) { pred = l < u ? u : l; }
        else { pred = l + u - ul; }
    }
    return a - pred;
}

// Block-wide exclusive scan (sum) of one value per thread; returns the
// exclusive prefix and writes the block total to *total.
template <typename T>
__device__ inline T block_exscan(T v, T* total, T* sm)
{
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= (uint32_t)d) { x += y; }
    }
    if (lane == 31u) { sm[wid] = x; }
    __syncthreads();
    if (wid == 0) {
        T s = lane < (blockDim.x >> 5) ? sm[lane] : (T)0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T y = __shfl_up_sync(0xFFFFFFFFu, s, d);
            if (lane >= (uint32_t)d) { s += y; }
        }
        sm[lane] = s;
    }
    __syncthreads();
    const T pre = (wid ? sm[wid - 1u] : (T)0) + x - v;
    *total = sm[(blockDim.x >> 5) - 1u];
    __syncthreads();
    return pre;
}

// One block per alpha band. Pass 1 computes the Rice parameters from the
// residual statistics, pass 2 emits (run, level) pairs and the trailing
// (run, 0) terminator with every code placed by a prefix sum of code lengths.
__global__ void __launch_bounds__(256) k_alpha(const ESlice* __restrict__ slices, const uint32_t* __restrict__ aslices,
                                               const EPlane* __restrict__ planes, const uint16_t* __restrict__ pix,
                                               uint8_t* __restrict__ stage, ESliceRes* __restrict__ sres,
                                               uint32_t* __restrict__ alpha_err)
{
    __shared__ unsigned long long sm64[32];
    __shared__ int32_t last_nz;
    __shared__ uint32_t kk[2];
    const uint32_t si = aslices[blockIdx.x];
    const ESlice& S = slices[si];
    const EPlane& P = planes[S.plane];
    const uint16_t* src = pix + P.pix_off;
    const uint32_t w = P.coded_w;
    const uint32_t py0 = S.y0 * 8u;
    const uint32_t count = w * S.bh * 8u;
    uint8_t* out = stage + S.stage_base;
    // max |source - near-lossless value| over the band (coded geometry)
    if (P.alpha_shift != 0u) {
        uint32_t me = 0;
        for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) {
            const uint32_t x = i % w, y = i / w;
            const uint32_t sx = min(x, P.vis_w - 1u), sy = min(py0 + y, P.vis_h - 1u);
            const uint32_t v = __ldg(src + (size_t)sy * P.vis_w + sx);
            const uint32_t q = alpha_sample(src, P, x, py0 + y);
            me = max(me, v > q ? v - q : q - v);
        }
        atomicMax(alpha_err + S.frame, me);
    }
    // pass 1: statistics
    unsigned long long s_lvl = 0, c_lvl = 0, s_run = 0, c_run = 0;
    if (threadIdx.x == 0) { last_nz = -1; }
    __syncthreads();
    for (uint32_t base = 0; base < count; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const int32_t r = i < count ? alpha_residual(src, P, py0, i) : 0;
        const bool nz = r != 0;
        // previous non-zero index: max over earlier non-zero lanes of this tile or the carry
        int32_t mine = nz ? (int32_t)i : -1;
        int32_t run_max = mine;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int32_t y = __shfl_up_sync(0xFFFFFFFFu, run_max, d);
            if ((threadIdx.x & 31u) >= (uint32_t)d) { run_max = max(run_max, y); }
        }
        __shared__ int32_t wmax[8];
        if ((threadIdx.x & 31u) == 31u) { wmax[threadIdx.x >> 5] = run_max; }
        __syncthreads();
        int32_t before = last_nz;
        for (uint32_t q = 0; q < (threadIdx.x >> 5); ++q) { before = max(before, wmax[q]); }
        const int32_t incl_prev = __shfl_up_sync(0xFFFFFFFFu, run_max, 1);
        if ((threadIdx.x & 31u) > 0u) { before = max(before, incl_prev); }
        if (nz) {
            s_run += (unsigned long long)((int32_t)i - before - 1);
            c_run++;
            s_lvl += map_s(r);
            c_lvl++;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1u) {
            int32_t m = last_nz;
            for (uint32_t q = 0; q < (blockDim.x >> 5); ++q) { m = max(m, wmax[q]); }
            last_nz = m;
        }
        __syncthreads();
    }
    unsigned long long tot;
    s_lvl = block_exscan<unsigned long long>(s_lvl, &tot, sm64); s_lvl = tot;
    c_lvl = block_exscan<unsigned long long>(c_lvl, &tot, sm64); c_lvl = tot;
    s_run = block_exscan<unsigned long long>(s_run, &tot, sm64); s_run = tot;
    c_run = block_exscan<unsigned long long>(c_run, &tot, sm64); c_run = tot;
    if (threadIdx.x == 0) {
        const int32_t tail = (int32_t)count - 1 - last_nz;
        if (tail > 0) { s_run += (unsigned long long)tail; c_run++; }
        uint32_t k1 = 0, k2 = 0;
        if (c_lvl != 0u && s_lvl != 0u) { const unsigned long long mn = s_lvl / c_lvl; while (k1 < 14u && (mn >> (k1 + 1u)) != 0u) { ++k1; } }
        if (c_run != 0u && s_run != 0u) { const unsigned long long mn = s_run / c_run; while (k2 < 14u && (mn >> (k2 + 1u)) != 0u) { ++k2; } }
        kk[0] = k1;
        kk[1] = k2;
        last_nz = -1;
    }
    __syncthreads();
    const uint32_t k1 = kk[0], k2 = kk[1];
    // pass 2: codes
    unsigned long long bitpos = 0;
    __shared__ unsigned long long carry_bits;
    if (threadIdx.x == 0) { carry_bits = 0; }
    __syncthreads();
    for (uint32_t base = 0; base < count; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const int32_t r = i < count ? alpha_residual(src, P, py0, i) : 0;
        const bool nz = r != 0;
        int32_t run_max = nz ? (int32_t)i : -1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int32_t y = __shfl_up_sync(0xFFFFFFFFu, run_max, d);
            if ((threadIdx.x & 31u) >= (uint32_t)d) { run_max = max(run_max, y); }
        }
        __shared__ int32_t wmax2[8];
        if ((threadIdx.x & 31u) == 31u) { wmax2[threadIdx.x >> 5] = run_max; }
        __syncthreads();
        int32_t before = last_nz;
        for (uint32_t q = 0; q < (threadIdx.x >> 5); ++q) { before = max(before, wmax2[q]); }
        const int32_t incl_prev = __shfl_up_sync(0xFFFFFFFFu, run_max, 1);
        if ((threadIdx.x & 31u) > 0u) { before = max(before, incl_prev); }
        const uint32_t run = nz ? (uint32_t)((int32_t)i - before - 1) : 0u;
        const uint32_t lm = nz ? map_s(r) : 0u;
        const unsigned long long len = nz ? (unsigned long long)(rice_len(k2, run) + rice_len(k1, lm)) : 0ull;
        unsigned long long tile_total;
        const unsigned long long pre = block_exscan<unsigned long long>(len, &tile_total, sm64);
        if (nz) {
            const unsigned long long o = carry_bits + pre;
            put_rice(out, o, k2, run);
            put_rice(out, o + rice_len(k2, run), k1, lm);
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1u) {
            int32_t m = last_nz;
            for (uint32_t q = 0; q < (blockDim.x >> 5); ++q) { m = max(m, wmax2[q]); }
            last_nz = m;
            carry_bits += tile_total;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        bitpos = carry_bits;
        const int32_t tail = (int32_t)count - 1 - last_nz;
        if (tail > 0) {
            put_rice(out, bitpos, k2, (uint32_t)tail);
            bitpos += rice_len(k2, (uint32_t)tail);
            put_rice(out, bitpos, k1, 0u);
            bitpos += rice_len(k1, 0u);
        }
        sres[si].nbytes = (uint32_t)((bitpos + 7u) >> 3);
        sres[si].plen = 0u;
        sres[si].xfin = (k1 << 8) | k2;  // alpha: Rice parameters for the slice header
    }
}

// ============================== packet assembly ==============================

__device__ __forceinline__ uint32_t payload_size(const ESlice& S, const ESliceRes& R)
{
    return S.kind == TCG_PLANE_COLOR ? (R.plen & 0xFFFFu) + 4u + R.nbytes : R.nbytes;
}

// one thread per frame: payload sizes, packet offsets, totals
__global__ void k_pack_sizes(const EFrame* __restrict__ frames, uint32_t nf, const ESlice* __restrict__ slices,
                             ESliceRes* __restrict__ sres, EFrameRes* __restrict__ fres)
{
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) { return; }
    const EFrame& F = frames[f];
    uint64_t off = 53u;
    uint32_t cp = 0, ap = 0, cs = 0, as = 0, err = 0;
    for (uint32_t i = 0; i < F.nslices; ++i) {
        const uint32_t si = F.slice0 + i;
        ESliceRes& R = sres[si];
        const uint32_t pay = payload_size(slices[si], R);
        R.payload = pay;
        R.pkt_off = off;
        off += 17u + pay;
        if (slices[si].kind == TCG_PLANE_COLOR) { cp += pay; cs++; } else { ap += pay; as++; }
        err |= R.err;
    }
    fres[f].size = off > 268435456ull ? 0xFFFFFFFFu : (uint32_t)off;
    fres[f].color_payload = cp;
    fres[f].alpha_payload = ap;
    fres[f].color_slices = cs;
    fres[f].alpha_slices = as;
    fres[f].err = err;
}

// grid (slice, part): copy prefix | state | stream (or the alpha bytes) into the packet
// Slice payloads into the packets: the prefix, the final coder state (4 bytes,
// big-endian) and the stream bytes. Each thread writes 4-byte aligned words of
// the destination; a word lying in the stream part takes its 4 bytes from the
// two aligned stream words that cover them, the rest go byte by byte.
__global__ void __launch_bounds__(256) k_pack_copy(const EFrame* __restrict__ frames, const ESlice* __restrict__ slices,
                                                   const ESliceRes* __restrict__ sres, const uint8_t* __restrict__ prefix,
                                                   const uint8_t* __restrict__ stage, uint8_t* __restrict__ pkt,
                                                   uint32_t cap_frames)
{
    const uint32_t si = blockIdx.x;
    const ESlice& S = slices[si];
    const ESliceRes& R = sres[si];
    const EFrame& F = frames[S.frame];
    uint8_t* dst = pkt + F.pkt_base + R.pkt_off + 17u;
    const uint32_t plen = S.kind == TCG_PLANE_COLOR ? (R.plen & 0xFFFFu) : 0u;
    const uint32_t head = S.kind == TCG_PLANE_COLOR ? plen + 4u : 0u;
    const uint8_t* stream = S.kind == TCG_PLANE_COLOR ? stage + S.stage_base + S.stage_cap - R.nbytes
                                                      : stage + S.stage_base;
    const uint32_t total = R.payload;
    const uint8_t* pre = prefix + (size_t)si * PREFIX_MAX;
    const uint32_t xfin = R.xfin;
    auto byte_at = [&](uint32_t i) -> uint8_t {
        if (i < plen) { return pre[i]; }
        if (i < head) { return (uint8_t)(xfin >> (8u * (3u - (i - plen)))); }
        return stream[i - head];
    };
    const uint32_t tid = blockIdx.y * blockDim.x + threadIdx.x, stride = gridDim.y * blockDim.x;
    const uint32_t lead = (uint32_t)((4u - ((uintptr_t)dst & 3u)) & 3u);  // bytes before the first aligned word
    const uint32_t nw = total > lead ? (total - lead) / 4u : 0u;
    const uint32_t tail0 = lead + 4u * nw;
    if (tid < lead && tid < total) { dst[tid] = byte_at(tid); }
    if (tail0 + tid < total) { dst[tail0 + tid] = byte_at(tail0 + tid); }  // at most 3 tail bytes
    uint32_t* dw = reinterpret_cast<uint32_t*>(dst + lead);
    for (uint32_t w = tid; w < nw; w += stride) {
        const uint32_t i = lead + 4u * w;
        uint32_t word;
        if (i >= head) {
            const uintptr_t sa = (uintptr_t)(stream + (i - head));
            const uint32_t* sw = reinterpret_cast<const uint32_t*>(sa & ~(uintptr_t)3);
            const uint32_t sh = (uint32_t)(sa & 3u);
            // the second word is read only when the 4 bytes straddle it (all are stream bytes)
            word = __byte_perm(sw[0], sh != 0u ? sw[1] : 0u, 0x3210u + sh * 0x1111u);
        } else {
            word = (uint32_t)byte_at(i) | ((uint32_t)byte_at(i + 1u) << 8) | ((uint32_t)byte_at(i + 2u) << 16) |
                   ((uint32_t)byte_at(i + 3u) << 24);
        }
        dw[w] = word;
    }
    (void)cap_frames;
}

// one block per slice: payload CRC-32 and the 17-byte slice header
__global__ void __launch_bounds__(256) k_pack_crc(const EFrame* __restrict__ frames, const ESlice* __restrict__ slices,
                                                  ESliceRes* __restrict__ sres, const uint32_t* __restrict__ crctab,
                                                  uint8_t* __restrict__ pkt)
{
    __shared__ uint32_t t[8 * 256];
    __shared__ uint32_t scratch[512];
    for (uint32_t i = threadIdx.x; i < 8u * 256u; i += blockDim.x) { t[i] = crctab[i]; }
    __syncthreads();
    const uint32_t si = blockIdx.x;
    const ESlice& S = slices[si];
    ESliceRes& R = sres[si];
    uint8_t* h = pkt + frames[S.frame].pkt_base + R.pkt_off;
    const uint32_t crc = crc32_block(h + 17u, R.payload, t, scratch);
    if (threadIdx.x == 0) {
        R.crc = crc;
        const uint32_t k1 = S.kind == TCG_PLANE_COLOR ? 0u : (R.xfin >> 8) & 0xFFu;
        const uint32_t k2 = S.kind == TCG_PLANE_COLOR ? 0u : R.xfin & 0xFFu;
        // 17-byte slice header (slice_map.c:7-20), big-endian
        h[0] = (uint8_t)(R.payload >> 24); h[1] = (uint8_t)(R.payload >> 16);
        h[2] = (uint8_t)(R.payload >> 8); h[3] = (uint8_t)R.payload;
        h[4] = (uint8_t)S.pidx;
        h[5] = (uint8_t)(S.y0 >> 8); h[6] = (uint8_t)S.y0;
        h[7] = (uint8_t)(S.bh >> 8); h[8] = (uint8_t)S.bh;
        h[9] = (uint8_t)S.qdb;
        h[10] = (uint8_t)k1; h[11] = (uint8_t)k2; h[12] = 0u;
        h[13] = (uint8_t)(crc >> 24); h[14] = (uint8_t)(crc >> 16);
        h[15] = (uint8_t)(crc >> 8); h[16] = (uint8_t)crc;
    }
}

// one thread per frame: header with the packet size, then CRC over bytes 0..48
__global__ void k_pack_header(const EFrame* __restrict__ frames, uint32_t nf, const EFrameRes* __restrict__ fres,
                              const uint32_t* __restrict__ crctab, uint8_t* __restrict__ pkt)
{
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) { return; }
    uint8_t* h = pkt + frames[f].pkt_base;
    const uint32_t size = fres[f].size;
    for (int i = 0; i < 53; ++i) { h[i] = frames[f].hdr[i]; }
    h[41] = (uint8_t)(size >> 24); h[42] = (uint8_t)(size >> 16); h[43] = (uint8_t)(size >> 8); h[44] = (uint8_t)size;
    uint32_t c = 0xFFFFFFFFu;
    for (int i = 0; i < 49; ++i) { c = crctab[(c ^ h[i]) & 0xFFu] ^ (c >> 8); }
    c ^= 0xFFFFFFFFu;
    h[49] = (uint8_t)(c >> 24); h[50] = (uint8_t)(c >> 16); h[51] = (uint8_t)(c >> 8); h[52] = (uint8_t)c;
}

// ============================ V8 segmented rANS ============================
//
// V8 (reference codec.c:3817-4320, layout packet.h:36-82) codes each colour
// plane as segments of sb = 8/16/32 consecutive blocks, each an independent
// rANS chain (DC predicted and DC context taken inside the segment only),
// grouped into tiles of tile_rows block rows that share one model chosen from
// their segments' summed counts. Per plane the packet holds
// [directory S x 12][tables T x 350][segment streams][tile CRCs T x 4].
// A 3840x2160 4:2:2 frame has 16,200 segments of ~3 K operations, so the
// chains run one lane each, 32 segments of a tile per warp sharing the
// tile's coding table in shared memory: the chains are short and many, and
// the encode is bound by issue and bandwidth instead of one long chain.
//
// Segments whose first block lies past the last tile's nominal block range
// belong to no tile; the reference leaves them unwritten and its self-check
// rejects the frame, and so does the host here (MALFORMED).

constexpr uint32_t V8_EXT = 8u, V8_DIR = 12u, V8_TABLE = 350u;

struct VSeg {
    uint32_t frame, plane, tile, nblk;   // tile = UINT32_MAX: in no tile (not coded)
    uint32_t blk0;                       // first global block
    uint32_t sidx;                       // index within the plane (directory entry)
    uint32_t qdb, pad;
    uint64_t op_base, stage_base, stage_cap;
};

struct VSegRes {
    uint32_t nops, nbytes, xfin, len;    // len: 4 + nbytes (0 when not coded)
    uint32_t rel;                        // stream offset from the plane's stream base
    uint32_t pad;
    uint64_t pkt_off;                    // stream offset from the packet start
};

struct VTile {
    uint32_t frame, plane, tidx, seg0, nseg, blk0, nblk, pad;
    uint64_t tab_off, str_off, str_bytes, crc_off;   // from the packet start (k_v8_sizes)
};

struct VPlaneD {
    uint32_t seg0, nseg, tile0, ntile;
    uint64_t dir_off, tab_off, str_off, crc_off;      // from the packet start (k_v8_sizes)
};

__device__ __forceinline__ uint32_t v8_block_dcm(const int32_t* coef, uint32_t gb, uint32_t i, uint32_t cols, bool* viol)
{
    const int32_t q0 = coef[(size_t)gb * 64u];
    const int32_t l = i > 0u ? coef[(size_t)(gb - 1u) * 64u] : 0;
    const int32_t t = i >= cols ? coef[(size_t)(gb - cols) * 64u] : 0;
    uint32_t dcm = map_s(q0 - dc_pred(i > 0u, l, i >= cols, t));
    if (dcm > 0x0FFFFFFFu) { dcm = 0x0FFFFFFFu; *viol = true; }
    return dcm;
}

// Tokens and tile histograms (codec.c:3882-3947, 2116-2151): a work item is a
// run of up to 256 blocks of one tile's segments; DC residuals and the DC
// context use the segment's own previous blocks only.
__global__ void __launch_bounds__(256) k_v8_tokens(const EWork* __restrict__ work, const VTile* __restrict__ tiles,
                                                   const EPlane* __restrict__ planes, const int32_t* __restrict__ coef,
                                                   const uint64_t* __restrict__ mask, uint32_t* __restrict__ dcm_out,
                                                   uint32_t* __restrict__ nops_out, uint32_t* __restrict__ hist,
                                                   ESliceRes* __restrict__ tres)
{
    extern __shared__ uint32_t sh[];  // [H_BINS][32] lane-replicated counters
    const EWork w = work[blockIdx.x];
    const VTile& T = tiles[w.slice];
    const EPlane& P = planes[T.plane];
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t i = threadIdx.x; i < H_BINS * 32u; i += blockDim.x) { sh[i] = 0u; }
    __syncthreads();
    bool viol = false;
    if (threadIdx.x < w.n) {
        const uint32_t gb = T.blk0 + w.lb0 + threadIdx.x;
        const uint32_t i = (gb - P.blk0) & ((1u << P.sb_log2) - 1u);
        const uint32_t dcm = v8_block_dcm(coef, gb, i, P.cols, &viol);
        const uint32_t dcc = bitlen32(dcm);
        uint32_t ctx = 0u;
        if (i > 0u) {
            bool dummy = false;
            ctx = dcp_ctx(bitlen32(v8_block_dcm(coef, gb - 1u, i - 1u, P.cols, &dummy)), true);
        }
        atomicAdd(&sh[(H_DC + dcc) * 32u + lane], 1u);
        atomicAdd(&sh[(H_JDC + ctx * DC_SYMS + dcc) * 32u + lane], 1u);
        uint32_t nops = 2u + suffix_chunks(dcc);
        const uint64_t m = mask[gb];
        uint32_t prev = 0u, pcat = 0u;
        bool has = false;
        int32_t cv[64];
        const int4* c4 = reinterpret_cast<const int4*>(coef + (size_t)gb * 64u);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int4 v = c4[k];
            cv[4 * k] = v.x; cv[4 * k + 1] = v.y; cv[4 * k + 2] = v.z; cv[4 * k + 3] = v.w;
        }
#pragma unroll
        for (uint32_t p = 1; p < 64u; ++p) {
            if (((m >> p) & 1u) == 0u) { continue; }
            uint32_t lm = map_s(cv[p]);
            if (lm > 0x07FFFFFFu) { lm = 0x07FFFFFFu; viol = true; }
            const uint32_t cat = bitlen32(lm);
            const uint32_t run = p - prev - 1u;
            atomicAdd(&sh[(H_RUN + run) * 32u + lane], 1u);
            atomicAdd(&sh[(H_LVL + cat) * 32u + lane], 1u);
            atomicAdd(&sh[(H_JPOS + pos_ctx(p) * LVL_SYMS + cat) * 32u + lane], 1u);
            atomicAdd(&sh[(H_JPREV + prev_ctx(pcat, has) * LVL_SYMS + cat) * 32u + lane], 1u);
            nops += 2u + suffix_chunks(cat);
            prev = p;
            pcat = cat;
            has = true;
        }
        atomicAdd(&sh[(H_RUN + 63u) * 32u + lane], 1u);
        dcm_out[gb] = dcm;
        nops_out[gb] = nops;
    }
    if (__syncthreads_or(viol) && threadIdx.x == 0) { atomicOr(&tres[w.slice].err, 1u); }
    uint32_t* g = hist + (size_t)w.slice * H_BINS;
    for (uint32_t b = threadIdx.x; b < H_BINS; b += blockDim.x) {
        uint32_t s = 0;
#pragma unroll 8
        for (uint32_t r = 0; r < 32u; ++r) { s += sh[b * 32u + ((r + b) & 31u)]; }
        if (s != 0u) { atomicAdd(&g[b], s); }
    }
}

// One warp per coded segment: operation offsets of its blocks in coding
// (reverse) order, the segment's count, identity padding to a multiple of 64.
__global__ void __launch_bounds__(256) k_v8_opscan(const VSeg* __restrict__ segs, const uint32_t* __restrict__ coded,
                                                   uint32_t ncoded, const uint32_t* __restrict__ nops,
                                                   uint32_t* __restrict__ opoff, uint32_t* __restrict__ ops,
                                                   VSegRes* __restrict__ sres)
{
    const uint32_t k = blockIdx.x * 8u + (threadIdx.x >> 5), lane = threadIdx.x & 31u;
    if (k >= ncoded) { return; }
    const uint32_t s = coded[k];
    const VSeg& S = segs[s];
    const uint32_t v = lane < S.nblk ? nops[S.blk0 + S.nblk - 1u - lane] : 0u;
    uint32_t x = v;
#pragma unroll
    for (uint32_t d = 1; d < 32u; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= d) { x += y; }
    }
    if (lane < S.nblk) { opoff[S.blk0 + S.nblk - 1u - lane] = x - v; }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, x, 31);
    if (lane == 0u) { sres[s].nops = total; }
    if (total + lane < ((total + 63u) & ~63u)) { ops[S.op_base + total + lane] = 0u; }
    if (total + 32u + lane < ((total + 63u) & ~63u)) { ops[S.op_base + total + 32u + lane] = 0u; }
}

// One warp per block (k_opgen's scheme), with the tile's models and the
// segment's own previous block as the DC context.
__global__ void __launch_bounds__(256) k_v8_opgen(const EWork* __restrict__ work, const VTile* __restrict__ tiles,
                                                  const EPlane* __restrict__ planes, const VSeg* __restrict__ segs,
                                                  const int32_t* __restrict__ coef, const uint64_t* __restrict__ mask,
                                                  const uint32_t* __restrict__ dcm, const uint32_t* __restrict__ opoff,
                                                  const ESliceRes* __restrict__ tres, uint32_t* __restrict__ ops)
{
    __shared__ uint8_t cats[8][64];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const EWork w = work[blockIdx.x];
    const uint32_t k = blockIdx.y * 8u + warp;
    if (k >= w.n) { return; }
    const VTile& T = tiles[w.slice];
    const EPlane& P = planes[T.plane];
    const uint32_t gb = T.blk0 + w.lb0 + k;
    const uint32_t lb = gb - P.blk0;
    const uint32_t i = lb & ((1u << P.sb_log2) - 1u);
    const VSeg& S = segs[P.seg0 + (lb >> P.sb_log2)];
    const uint32_t pl = tres[w.slice].plen;
    const uint32_t lmod = (pl >> 16) & 3u, dmod = (pl >> 20) & 1u;
    uint32_t* o = ops + S.op_base + opoff[gb];
    const int32_t* c = coef + (size_t)gb * 64u;
    const uint64_t m = mask[gb];
    uint32_t lmv[2], cat[2], cnt[2];
#pragma unroll
    for (uint32_t h = 0; h < 2u; ++h) {
        const uint32_t p = lane + 32u * h;
        const bool nz = ((m >> p) & 1u) != 0u;
        const uint32_t lv = nz ? map_s(c[p]) : 0u;
        lmv[h] = lv > 0x07FFFFFFu ? 0x07FFFFFFu : lv;
        cat[h] = nz ? bitlen32(lmv[h]) : 0u;
        cnt[h] = nz ? 2u + suffix_chunks(cat[h]) : 0u;
        cats[warp][p] = (uint8_t)cat[h];
    }
    const uint32_t packed = cnt[0] | (cnt[1] << 16);
    uint32_t incl = packed;
#pragma unroll
    for (uint32_t d = 1; d < 32u; d <<= 1) {
        const uint32_t t = __shfl_down_sync(0xFFFFFFFFu, incl, d);
        if (lane + d < 32u) { incl += t; }
    }
    const uint32_t above = incl - packed;
    const uint32_t all = __shfl_sync(0xFFFFFFFFu, incl, 0);
    const uint32_t hi_total = all >> 16, total = (all & 0xFFFFu) + hi_total;
    __syncwarp();
#pragma unroll
    for (uint32_t h = 0; h < 2u; ++h) {
        if (cnt[h] == 0u) { continue; }
        const uint32_t p = lane + 32u * h;
        uint32_t* q = o + 1u + (h ? (above >> 16) : hi_total + (above & 0xFFFFu));
        const uint64_t lower = m & ((1ull << p) - 1ull);
        const uint32_t below = lower != 0u ? 63u - (uint32_t)__clzll((long long)lower) : 0u;
        put_suffix_ops(q, cat[h], lmv[h]);
        uint32_t ctx = 0u;
        if (lmod == 1u) {
            ctx = pos_ctx(p);
        } else if (lmod == 2u) {
            ctx = prev_ctx(lower != 0u ? cats[warp][below] : 0u, lower != 0u);
        }
        *q++ = op_sym(T_LVL + ctx * LVL_SYMS + cat[h]);
        *q = op_sym(T_RUN + (p - below - 1u));
    }
    if (lane == 0u) {
        o[0] = op_sym(T_RUN + 63u);
        uint32_t* q = o + 1u + total;
        const uint32_t dm = dcm[gb];
        const uint32_t ds = bitlen32(dm);
        put_suffix_ops(q, ds, dm);
        const uint32_t dctx = dmod ? dcp_ctx(i > 0u ? bitlen32(dcm[gb - 1u]) : 0u, i > 0u) : 0u;
        *q = op_sym(T_DC + dctx * DC_SYMS + ds);
    }
}

// One lane per segment, 32 segments of one tile per warp: the warp expands
// the tile's coding table into shared memory once, then every lane runs its
// segment's backward chain as k_chain does.
constexpr size_t V8CH_SMEM = (size_t)OP_ENTRIES * sizeof(uint4);

__global__ void __launch_bounds__(32) k_v8_chain(const VSeg* __restrict__ segs, const int32_t* __restrict__ lanes,
                                                 const uint32_t* __restrict__ ctile, const uint32_t* __restrict__ ops,
                                                 const uint32_t* __restrict__ stab, const uint32_t* __restrict__ div_m,
                                                 const uint8_t* __restrict__ div_l, uint8_t* __restrict__ stage,
                                                 VSegRes* __restrict__ sres)
{
    extern __shared__ uint4 chain_tab[];
    const uint32_t lane = threadIdx.x;
    const uint32_t* st = stab + (size_t)ctile[blockIdx.x] * T_SIZE;
    for (uint32_t w = lane; w < OP_ENTRIES; w += 32u) {
        chain_tab[w] = w < OP_CHUNKS ? chunk_entry(w) : symbol_entry(__ldg(st + (w - OP_CHUNKS)), div_m, div_l);
    }
    __syncwarp();
    const int32_t si = lanes[blockIdx.x * 32u + lane];
    if (si < 0) { return; }
    const uint4* tab = chain_tab;
    const VSeg& S = segs[si];
    const uint32_t nops = sres[si].nops;
    const uint4* op4 = reinterpret_cast<const uint4*>(ops + S.op_base);
    uint8_t* const end = stage + S.stage_base + S.stage_cap;
    uint8_t* p = end;
    uint32_t x = RANS_L;
    // sixteen groups (64 operations) in registers, each reloaded sixteen groups
    // ahead of its use (the segments' chains are short and many, so more loads
    // in flight pay here: 17.6 against 18.3 ms for 60 3840x2160 frames)
    uint4 q0 = op_group(op4, 0u, nops), q1 = op_group(op4, 1u, nops), q2 = op_group(op4, 2u, nops);
    uint4 q3 = op_group(op4, 3u, nops), q4 = op_group(op4, 4u, nops), q5 = op_group(op4, 5u, nops);
    uint4 q6 = op_group(op4, 6u, nops), q7 = op_group(op4, 7u, nops), q8 = op_group(op4, 8u, nops);
    uint4 q9 = op_group(op4, 9u, nops), q10 = op_group(op4, 10u, nops), q11 = op_group(op4, 11u, nops);
    uint4 q12 = op_group(op4, 12u, nops), q13 = op_group(op4, 13u, nops), q14 = op_group(op4, 14u, nops);
    uint4 q15 = op_group(op4, 15u, nops);
    for (uint32_t g = 0; 4u * g < nops; g += 16u) {
        ENC_GROUP(q0); q0 = op_group(op4, g + 16u, nops);
        ENC_GROUP(q1); q1 = op_group(op4, g + 17u, nops);
        ENC_GROUP(q2); q2 = op_group(op4, g + 18u, nops);
        ENC_GROUP(q3); q3 = op_group(op4, g + 19u, nops);
        ENC_GROUP(q4); q4 = op_group(op4, g + 20u, nops);
        ENC_GROUP(q5); q5 = op_group(op4, g + 21u, nops);
        ENC_GROUP(q6); q6 = op_group(op4, g + 22u, nops);
        ENC_GROUP(q7); q7 = op_group(op4, g + 23u, nops);
        ENC_GROUP(q8); q8 = op_group(op4, g + 24u, nops);
        ENC_GROUP(q9); q9 = op_group(op4, g + 25u, nops);
        ENC_GROUP(q10); q10 = op_group(op4, g + 26u, nops);
        ENC_GROUP(q11); q11 = op_group(op4, g + 27u, nops);
        ENC_GROUP(q12); q12 = op_group(op4, g + 28u, nops);
        ENC_GROUP(q13); q13 = op_group(op4, g + 29u, nops);
        ENC_GROUP(q14); q14 = op_group(op4, g + 30u, nops);
        ENC_GROUP(q15); q15 = op_group(op4, g + 31u, nops);
    }
    sres[si].nbytes = (uint32_t)(end - p);
    sres[si].xfin = x;
}

// One block per frame: segment stream offsets (a block-wide scan per plane),
// plane section offsets, tile table / stream / CRC ranges, the packet size,
// the 8-byte extension header; token-domain errors of its tiles.
__global__ void __launch_bounds__(1024) k_v8_sizes(const EFrame* __restrict__ frames, VPlaneD* __restrict__ vp,
                                                   const VSeg* __restrict__ segs, VSegRes* __restrict__ sres,
                                                   VTile* __restrict__ tiles, const ESliceRes* __restrict__ tres,
                                                   EFrameRes* __restrict__ fres, uint8_t* __restrict__ pkt,
                                                   const uint8_t* __restrict__ ext)
{
    __shared__ unsigned long long sm[32];
    const EFrame& F = frames[blockIdx.x];
    uint64_t off = 53u + V8_EXT;
    uint32_t err = 0u;
    for (uint32_t pi = 0; pi < F.nslices; ++pi) {
        VPlaneD& P = vp[F.slice0 + pi];
        const uint64_t dir = off, tab = dir + (uint64_t)P.nseg * V8_DIR, str = tab + (uint64_t)P.ntile * V8_TABLE;
        unsigned long long carry = 0;
        for (uint32_t b = 0; b < P.nseg; b += blockDim.x) {
            const uint32_t k = b + threadIdx.x;
            const uint32_t s = P.seg0 + k;
            const uint32_t len = k < P.nseg && segs[s].tile != 0xFFFFFFFFu ? 4u + sres[s].nbytes : 0u;
            unsigned long long tot;
            const unsigned long long pre = block_exscan<unsigned long long>(len, &tot, sm);
            if (k < P.nseg) {
                sres[s].len = len;
                sres[s].rel = (uint32_t)(carry + pre);
                sres[s].pkt_off = str + carry + pre;
            }
            carry += tot;
        }
        const uint64_t crc = str + carry;
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < P.ntile; t += blockDim.x) {
            VTile& T = tiles[P.tile0 + t];
            T.tab_off = tab + (uint64_t)t * V8_TABLE;
            T.crc_off = crc + 4u * t;
            if (T.nseg != 0u) {
                const VSegRes& a = sres[T.seg0];
                const VSegRes& z = sres[T.seg0 + T.nseg - 1u];
                T.str_off = a.pkt_off;
                T.str_bytes = z.pkt_off + z.len - a.pkt_off;
            } else {
                T.str_off = str;
                T.str_bytes = 0u;
            }
            err |= tres[P.tile0 + t].err;
        }
        if (threadIdx.x == 0) {
            P.dir_off = dir;
            P.tab_off = tab;
            P.str_off = str;
            P.crc_off = crc;
        }
        off = crc + 4u * P.ntile;
    }
    err = __syncthreads_or(err != 0u) ? 1u : 0u;
    if (threadIdx.x == 0) {
        fres[blockIdx.x].size = off > 0x10000000ull ? 0xFFFFFFFFu : (uint32_t)off;
        fres[blockIdx.x].color_payload = (uint32_t)(off - 53u - V8_EXT);
        fres[blockIdx.x].alpha_payload = 0u;
        fres[blockIdx.x].err = err;
        fres[blockIdx.x].color_slices = 0u;
        fres[blockIdx.x].alpha_slices = 0u;
    }
    if (threadIdx.x < V8_EXT) { pkt[F.pkt_base + 53u + threadIdx.x] = ext[blockIdx.x * V8_EXT + threadIdx.x]; }
}

// One warp per segment: its directory entry and its stream (final state
// big-endian, then the bytes the chain emitted) at the offsets k_v8_sizes set.
__global__ void __launch_bounds__(256) k_v8_copy(const EFrame* __restrict__ frames, const VPlaneD* __restrict__ vp,
                                                 const VSeg* __restrict__ segs, uint32_t nseg,
                                                 const VSegRes* __restrict__ sres, const uint8_t* __restrict__ stage,
                                                 uint8_t* __restrict__ pkt)
{
    const uint32_t s = blockIdx.x * 8u + (threadIdx.x >> 5), lane = threadIdx.x & 31u;
    if (s >= nseg) { return; }
    const VSeg& S = segs[s];
    const VSegRes& R = sres[s];
    const EFrame& F = frames[S.frame];
    const VPlaneD& P = vp[S.plane];
    uint8_t* de = pkt + F.pkt_base + P.dir_off + (uint64_t)S.sidx * V8_DIR;
    if (lane < V8_DIR) {
        const bool coded = S.tile != 0xFFFFFFFFu;
        uint32_t b = 0u;
        if (coded) {
            if (lane < 4u) { b = (R.rel >> (8u * (3u - lane))) & 0xFFu; }
            else if (lane < 8u) { b = (R.len >> (8u * (7u - lane))) & 0xFFu; }
            else if (lane == 8u) { b = S.qdb; }
        }
        de[lane] = (uint8_t)b;
    }
    if (S.tile == 0xFFFFFFFFu) { return; }
    uint8_t* dst = pkt + F.pkt_base + R.pkt_off;
    const uint8_t* stream = stage + S.stage_base + S.stage_cap - R.nbytes;
    const uint32_t total = R.len, xfin = R.xfin;
    auto byte_at = [&](uint32_t i) -> uint8_t {
        return i < 4u ? (uint8_t)(xfin >> (8u * (3u - i))) : stream[i - 4u];
    };
    const uint32_t lead = (uint32_t)((4u - ((uintptr_t)dst & 3u)) & 3u);
    const uint32_t nw = total > lead ? (total - lead) / 4u : 0u;
    const uint32_t tail0 = lead + 4u * nw;
    if (lane < lead && lane < total) { dst[lane] = byte_at(lane); }
    if (tail0 + lane < total) { dst[tail0 + lane] = byte_at(tail0 + lane); }
    uint32_t* dw = reinterpret_cast<uint32_t*>(dst + lead);
    for (uint32_t w = lane; w < nw; w += 32u) {
        const uint32_t i = lead + 4u * w;
        uint32_t word;
        if (i >= 4u) {
            const uintptr_t sa = (uintptr_t)(stream + (i - 4u));
            const uint32_t* sw = reinterpret_cast<const uint32_t*>(sa & ~(uintptr_t)3);
            const uint32_t sh = (uint32_t)(sa & 3u);
            word = __byte_perm(sw[0], sh != 0u ? sw[1] : 0u, 0x3210u + sh * 0x1111u);
        } else {
            word = (uint32_t)byte_at(i) | ((uint32_t)byte_at(i + 1u) << 8) | ((uint32_t)byte_at(i + 2u) << 16) |
                   ((uint32_t)byte_at(i + 3u) << 24);
        }
        dw[w] = word;
    }
}

// One block per tile: the 350-byte table (flags, five DC rows, run row, five
// level rows; rows past the model's contexts are the all-zero row {1, 0, ...},
// codec.c:3949-3971), then the CRC of the table and the member streams.
__global__ void __launch_bounds__(256) k_v8_tiles(const EFrame* __restrict__ frames, const VTile* __restrict__ tiles,
                                                  const ESliceRes* __restrict__ tres, const uint8_t* __restrict__ prefix,
                                                  const uint32_t* __restrict__ crctab, uint8_t* __restrict__ pkt)
{
    __shared__ uint32_t t[8 * 256];
    __shared__ uint32_t scratch[512];
    __shared__ uint32_t crc_tab;
    for (uint32_t i = threadIdx.x; i < 8u * 256u; i += blockDim.x) { t[i] = crctab[i]; }
    const uint32_t ti = blockIdx.x;
    const VTile& T = tiles[ti];
    uint8_t* base = pkt + frames[T.frame].pkt_base;
    const uint32_t pl = tres[ti].plen;
    const uint32_t lm = (pl >> 16) & 3u, dm = (pl >> 20) & 1u;
    const uint32_t nd = dm ? DCP_CTX : 1u, nl = lm == 1u ? POS_CTX : lm == 2u ? PREV_CTX : 1u;
    const uint8_t* pre = prefix + (size_t)ti * PREFIX_MAX;
    uint8_t* tb = base + T.tab_off;
    for (uint32_t k = threadIdx.x; k < V8_TABLE; k += blockDim.x) {
        uint8_t v;
        if (k == 0u) {
            v = pre[0];
        } else if (k < 1u + DCP_CTX * DC_SYMS) {
            const uint32_t c = (k - 1u) / DC_SYMS, j = (k - 1u) % DC_SYMS;
            v = c < nd ? pre[1u + c * DC_SYMS + j] : (uint8_t)(j == 0u);
        } else if (k < 1u + DCP_CTX * DC_SYMS + RUN_SYMS) {
            v = pre[1u + nd * DC_SYMS + (k - 1u - DCP_CTX * DC_SYMS)];
        } else {
            const uint32_t r = k - 1u - DCP_CTX * DC_SYMS - RUN_SYMS, c = r / LVL_SYMS, j = r % LVL_SYMS;
            v = c < nl ? pre[1u + nd * DC_SYMS + RUN_SYMS + c * LVL_SYMS + j] : (uint8_t)(j == 0u);
        }
        tb[k] = v;
    }
    __syncthreads();
    const uint32_t c1 = crc32_block(tb, V8_TABLE, t, scratch);
    if (threadIdx.x == 0) { crc_tab = c1; }
    __syncthreads();
    const uint32_t c2 = crc32_block(base + T.str_off, T.str_bytes, t, scratch);
    if (threadIdx.x == 0) {
        const uint32_t c = T.str_bytes == 0u ? crc_tab : crc_combine(crc_tab, c2, gf2_xpow8n(T.str_bytes));
        uint8_t* h = base + T.crc_off;
        h[0] = (uint8_t)(c >> 24); h[1] = (uint8_t)(c >> 16); h[2] = (uint8_t)(c >> 8); h[3] = (uint8_t)c;
    }
}

// ================================== driver ==================================

static size_t align_up(size_t v, size_t a) { return (v + a - 1u) / a * a; }


// Enqueue one batch on the context's streams: descriptors, sample copies,
// kernels and the copy of the per-frame results to pinned host memory. The
// sample copies start after `after` (when given) and C->gate is recorded
// behind them. ef receives the frame table encode_results needs.
static int32_t encode_launch(Ctx* C, const tcg_enc_frame* frames, uint32_t count, cudaEvent_t after,
                             std::vector<EFrame>& ef)
{
    // ---------------- host planning ----------------
    std::vector<EPlane> planes;
    std::vector<ESlice> slices;
    ef.assign(count, EFrame());
    std::vector<uint32_t> cplanes, cslices, aslices;
    std::vector<EWork> work;
    uint64_t pix_elems = 0, nblk = 0, ops_words = 0, stage_bytes = 0, pkt_bytes = 0;
    for (uint32_t f = 0; f < count; ++f) {
        const tcg_enc_frame& F = frames[f];
        ef[f].slice0 = (uint32_t)slices.size();
        ef[f].nslices = 0;
        memset(ef[f].hdr, 0, sizeof(ef[f].hdr));
        memcpy(ef[f].hdr, F.header, 53);
        uint64_t fbound = 53;
        for (uint32_t p = 0; p < F.planes; ++p) {
            const tcg_enc_plane& I = F.plane[p];
            EPlane P;
            memset(&P, 0, sizeof(P));
            P.pix_off = pix_elems;
            pix_elems += (uint64_t)I.vis_w * I.vis_h;
            pix_elems = align_up(pix_elems, 64);
            P.vis_w = I.vis_w; P.vis_h = I.vis_h; P.coded_w = I.coded_w; P.coded_h = I.coded_h;
            P.cols = I.cols; P.rows = I.rows; P.kind = I.kind; P.alpha_shift = I.alpha_shift;
            P.bd = F.bit_depth;
            P.blk0 = (uint32_t)nblk;
            P.fclamp = I.fclamp;
            P.q_is_one = 1u;
            for (int i = 0; i < 64; ++i) {
                P.Q[i] = I.Q[i];
                if (I.Q[i] != 1u) { P.q_is_one = 0u; }
                div_magic(I.Q[i] != 0u ? I.Q[i] : 1u, &P.Qm[i], &P.Qsh[i]);
            }
            const uint32_t pg = (uint32_t)planes.size();
            if (I.kind == TCG_PLANE_COLOR) {
                cplanes.push_back(pg);
                nblk += (uint64_t)I.cols * I.rows;
            }
            for (uint32_t y0 = 0; y0 < I.rows; y0 += F.slice_rows) {
                ESlice S;
                memset(&S, 0, sizeof(S));
                S.frame = f; S.plane = pg; S.kind = I.kind; S.pidx = p;
                S.y0 = y0; S.bh = std::min(F.slice_rows, I.rows - y0); S.cols = I.cols;
                S.qdb = I.qdb;
                uint64_t pay;
                if (I.kind == TCG_PLANE_COLOR) {
                    S.blk0 = P.blk0 + y0 * I.cols;
                    S.nblk = S.bh * I.cols;
                    S.op_base = ops_words;
                    // at most 256 operations per block, then 256 words for the
                    // identity padding and look-ahead reads of the chain
                    ops_words += (uint64_t)S.nblk * 256u + 256u;
                    S.stage_cap = (uint64_t)S.nblk * 512u + 64u;
                    pay = PREFIX_MAX + 4u + S.stage_cap;
                    const uint32_t si = (uint32_t)slices.size();
                    cslices.push_back(si);
                    for (uint32_t lb = 0; lb < S.nblk; lb += 256u) {
                        EWork w = {si, lb, std::min(256u, S.nblk - lb), 0u};
                        work.push_back(w);
                    }
                } else {
                    S.stage_cap = (uint64_t)I.coded_w * S.bh * 8u * 16u + 64u;
                    pay = S.stage_cap;
                    aslices.push_back((uint32_t)slices.size());
                }
                S.stage_base = stage_bytes;
                stage_bytes = align_up(stage_bytes + S.stage_cap, 256);
                fbound += 17u + pay;
                slices.push_back(S);
                ef[f].nslices++;
            }
            planes.push_back(P);
        }
        ef[f].pkt_base = pkt_bytes;
        pkt_bytes = align_up(pkt_bytes + fbound, 256);
    }
    const uint32_t ns = (uint32_t)slices.size(), nc = (uint32_t)cslices.size();
    // chain lanes: largest slices first so each warp holds similar chain lengths
    std::vector<uint32_t> order = cslices;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return slices[a].nblk > slices[b].nblk; });

    // ---------------- device buffers ----------------
    const size_t desc_bytes = align_up(planes.size() * sizeof(EPlane), 256) + align_up(ns * sizeof(ESlice), 256) +
                              align_up(count * sizeof(EFrame), 256) + align_up(work.size() * sizeof(EWork), 256) +
                              align_up((cplanes.size() + cslices.size() + aslices.size() + order.size()) * 4u + 16u, 256) +
                              align_up(cplanes.size() * 4u + 16u, 256) + 1024u;
    if (!dreserve(C, B_PIX, pix_elems * 2u + 256) || !dreserve(C, B_COEF, nblk * 256u + 256) ||
        !dreserve(C, B_UMAP, (nblk + 31u) / 32u * 4u + 256) ||
        !dreserve(C, B_MASK, nblk * 8u + 256) || !dreserve(C, B_DCM, nblk * 4u + 256) ||
        !dreserve(C, B_NOPS, nblk * 4u + 256) || !dreserve(C, B_OPOFF, nblk * 4u + 256) ||
        !dreserve(C, B_HIST, (size_t)ns * H_BINS * 4u + 256) || !dreserve(C, B_STAB, (size_t)ns * T_SIZE * 4u + 256) ||
        !dreserve(C, B_TMP0, (size_t)ns * PREFIX_MAX + 256) || !dreserve(C, B_OPS, ops_words * 4u + 256) ||
        !dreserve(C, B_STAGE, stage_bytes + 256) || !dreserve(C, B_SRES, (size_t)ns * sizeof(ESliceRes) + 256) ||
        !dreserve(C, B_FRES, (size_t)count * (sizeof(EFrameRes) + 4u) + 256) || !dreserve(C, B_PKT, pkt_bytes + 256) ||
        !dreserve(C, B_DESC, desc_bytes) || !hreserve(C, 0, desc_bytes) ||
        !hreserve(C, 1, (size_t)count * sizeof(EFrameRes) + 4096)) {
        return TCG_ERR_OUT_OF_MEMORY;
    }
    cudaStream_t st = C->stream;
    // descriptors through pinned staging
    uint8_t* hd = (uint8_t*)C->h[0].p;
    uint8_t* dd = dptr<uint8_t>(C, B_DESC);
    size_t o = 0;
    auto put = [&](const void* src, size_t n) -> size_t {
        const size_t at = o;
        if (n) { memcpy(hd + o, src, n); }
        o = align_up(o + n, 256);
        return at;
    };
    const size_t o_pl = put(planes.data(), planes.size() * sizeof(EPlane));
    const size_t o_sl = put(slices.data(), ns * sizeof(ESlice));
    const size_t o_fr = put(ef.data(), count * sizeof(EFrame));
    const size_t o_wk = put(work.data(), work.size() * sizeof(EWork));
    const size_t o_cp = put(cplanes.data(), cplanes.size() * 4u);
    const size_t o_cs = put(cslices.data(), cslices.size() * 4u);
    const size_t o_as = put(aslices.data(), aslices.size() * 4u);
    const size_t o_or = put(order.data(), order.size() * 4u);
    std::vector<uint32_t> pstart(cplanes.size());  // first block of each colour plane (unit lookup)
    for (size_t i = 0; i < cplanes.size(); ++i) { pstart[i] = planes[cplanes[i]].blk0; }
    const size_t o_ps = put(pstart.data(), pstart.size() * 4u);
    call_begin(C);
    TCG_CHECK(cudaMemcpyAsync(dd, hd, o, cudaMemcpyHostToDevice, st));
    const EPlane* d_pl = (const EPlane*)(dd + o_pl);
    const ESlice* d_sl = (const ESlice*)(dd + o_sl);
    const EFrame* d_fr = (const EFrame*)(dd + o_fr);
    const EWork* d_wk = (const EWork*)(dd + o_wk);
    const uint32_t* d_cp = (const uint32_t*)(dd + o_cp);
    const uint32_t* d_cs = (const uint32_t*)(dd + o_cs);
    const uint32_t* d_as = (const uint32_t*)(dd + o_as);
    const uint32_t* d_or = (const uint32_t*)(dd + o_or);
    const uint32_t* d_ps = (const uint32_t*)(dd + o_ps);

    // samples: one 2-D copy per plane (host or device source, caller stride)
    uint16_t* d_pix = dptr<uint16_t>(C, B_PIX);
    if (after != nullptr) { TCG_CHECK(cudaStreamWaitEvent(st, after, 0)); }
    {
        uint32_t pg = 0;
        for (uint32_t f = 0; f < count; ++f) {
            for (uint32_t p = 0; p < frames[f].planes; ++p, ++pg) {
                const tcg_enc_plane& I = frames[f].plane[p];
                if (I.stride == I.vis_w) {  // tight rows: one flat copy
                    TCG_CHECK(cudaMemcpyAsync(d_pix + planes[pg].pix_off, I.src, (size_t)I.vis_w * I.vis_h * 2u,
                                              cudaMemcpyDefault, st));
                } else {
                    TCG_CHECK(cudaMemcpy2DAsync(d_pix + planes[pg].pix_off, (size_t)I.vis_w * 2u, I.src,
                                                I.stride * 2u, (size_t)I.vis_w * 2u, I.vis_h, cudaMemcpyDefault, st));
                }
            }
        }
    }
    TCG_CHECK(cudaEventRecord(C->gate, st));
    ESliceRes* d_sres = dptr<ESliceRes>(C, B_SRES);
    EFrameRes* d_fres = dptr<EFrameRes>(C, B_FRES);
    uint32_t* d_aerr = reinterpret_cast<uint32_t*>(dptr<uint8_t>(C, B_FRES) + align_up(count * sizeof(EFrameRes), 16));
    TCG_CHECK(cudaMemsetAsync(d_sres, 0, (size_t)ns * sizeof(ESliceRes), st));
    TCG_CHECK(cudaMemsetAsync(d_aerr, 0, (size_t)count * 4u, st));
    TCG_CHECK(cudaMemsetAsync(dptr<uint32_t>(C, B_HIST), 0, (size_t)ns * H_BINS * 4u, st));
    const DevTables& T = tables();
    int32_t* d_coef = dptr<int32_t>(C, B_COEF);
    uint64_t* d_mask = dptr<uint64_t>(C, B_MASK);
    uint32_t* d_dcm = dptr<uint32_t>(C, B_DCM);
    uint32_t* d_nops = dptr<uint32_t>(C, B_NOPS);
    uint32_t* d_opoff = dptr<uint32_t>(C, B_OPOFF);
    uint32_t* d_hist = dptr<uint32_t>(C, B_HIST);
    uint32_t* d_stab = dptr<uint32_t>(C, B_STAB);
    uint8_t* d_prefix = dptr<uint8_t>(C, B_TMP0);
    uint32_t* d_ops = dptr<uint32_t>(C, B_OPS);
    uint8_t* d_stage = dptr<uint8_t>(C, B_STAGE);
    uint8_t* d_pkt = dptr<uint8_t>(C, B_PKT);

    if (!aslices.empty()) {
        // Alpha slices (MED residuals, Rice pairs) read only the samples and write
        // only their own staging windows and results, so they run on a third
        // stream beside the colour path; the stream rejoins before packing.
        cudaStream_t as = aux_stream(C);
        if (as == nullptr) { return TCG_ERR_OUT_OF_MEMORY; }
        TCG_CHECK(cudaEventRecord(C->afork, st));
        TCG_CHECK(cudaStreamWaitEvent(as, C->afork, 0));
        for (uint32_t a : aslices) {
            TCG_CHECK(cudaMemsetAsync(d_stage + slices[a].stage_base, 0, slices[a].stage_cap, as));
        }
        TCG_LAUNCH_ON(C, as, K_ALPHA, k_alpha, (uint32_t)aslices.size(), 256, 0, d_sl, d_as, d_pl, d_pix, d_stage,
                      d_sres, d_aerr);
        TCG_CHECK(cudaEventRecord(C->ajoin, as));
    }
    if (nblk > 0) {
        bool any_wide = false;
        for (uint32_t pg : cplanes) { any_wide = any_wide || planes[pg].bd > 12u; }
        uint32_t* d_umap = dptr<uint32_t>(C, B_UMAP);
        TCG_LAUNCH(C, K_UNIT_MAP, k_unit_map, (uint32_t)((nblk + 8191u) / 8192u), 256, 0, d_ps, 1u,
                   (uint32_t)cplanes.size(), (uint32_t)nblk, d_umap);
        TCG_LAUNCH(C, K_FDCT, k_fdct, (uint32_t)((nblk + FB_BLOCKS - 1u) / FB_BLOCKS), 256, 0, d_pl, d_cp,
                   (uint32_t)cplanes.size(), (uint32_t)nblk, d_pix, d_coef, d_mask, d_ps, d_umap);
        if (any_wide) {
            TCG_LAUNCH(C, K_FDCT, k_fdct_wide, (uint32_t)((nblk + 127u) / 128u), 128, 0, d_pl, d_cp,
                       (uint32_t)cplanes.size(), (uint32_t)nblk, d_pix, d_coef, d_mask);
        }
        const size_t tok_smem = H_BINS * 32u * 4u;
        static bool attr_set = false;
        if (!attr_set) {
            cudaFuncSetAttribute(k_tokens, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tok_smem);
            attr_set = true;
        }
        TCG_LAUNCH(C, K_TOKENS, k_tokens, (uint32_t)work.size(), 256, tok_smem, d_wk, d_sl, d_coef, d_mask, d_dcm, d_nops,
                   d_hist, d_sres);
        TCG_LAUNCH(C, K_SELECT, k_select, nc, 32, 0, d_sl, d_cs, d_hist, T.log2, d_stab, d_prefix, d_sres);
        TCG_LAUNCH(C, K_OPSCAN, k_opscan, nc, 1024, 0, d_sl, d_cs, d_nops, d_opoff, d_ops, d_sres);
        TCG_LAUNCH(C, K_OPGEN, k_opgen, dim3((uint32_t)work.size(), 32), 256, 0, d_wk, d_sl, d_coef, d_mask, d_dcm,
                   d_opoff, d_sres, d_ops);
        static bool chain_attr = false;
        if (!chain_attr) {
            cudaFuncSetAttribute(k_chain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CHAIN_SMEM);
            chain_attr = true;
        }
        TCG_LAUNCH(C, K_CHAIN, k_chain, (nc + CHAIN_LANES - 1u) / CHAIN_LANES, CHAIN_LANES, CHAIN_SMEM, d_sl, d_or, nc,
                   d_ops, d_stab, T.div_m, T.div_l, d_stage, d_sres);
    }
    if (!aslices.empty()) {
        // the alpha slices have been on their own stream since the samples arrived
        TCG_CHECK(cudaStreamWaitEvent(st, C->ajoin, 0));
    }
    TCG_LAUNCH(C, K_PACK_SIZES, k_pack_sizes, (count + 127u) / 128u, 128, 0, d_fr, count, d_sl, d_sres, d_fres);
    TCG_LAUNCH(C, K_PACK_COPY, k_pack_copy, dim3(ns, 8), 256, 0, d_fr, d_sl, d_sres, d_prefix, d_stage, d_pkt, count);
    TCG_LAUNCH(C, K_PACK_CRC, k_pack_crc, ns, 256, 0, d_fr, d_sl, d_sres, T.crc, d_pkt);
    TCG_LAUNCH(C, K_PACK_HEADER, k_pack_header, (count + 127u) / 128u, 128, 0, d_fr, count, d_fres, T.crc, d_pkt);
    TCG_CHECK(cudaGetLastError());

    // ---------------- results ----------------
    EFrameRes* hf = (EFrameRes*)C->h[1].p;
    uint32_t* ha = (uint32_t*)((uint8_t*)C->h[1].p + align_up(count * sizeof(EFrameRes), 16));
    TCG_CHECK(cudaMemcpyAsync(hf, d_fres, count * sizeof(EFrameRes), cudaMemcpyDeviceToHost, st));
    TCG_CHECK(cudaMemcpyAsync(ha, d_aerr, count * 4u, cudaMemcpyDeviceToHost, st));
    return 0;
}

// V8 batch: every frame of the call is V8 (tcg_encode splits mixed batches).
// Host planning lays out planes, segments, tiles, token work items and the
// chain warps (32 segments of one tile each); the device does the rest.
static int32_t encode_launch_v8(Ctx* C, const tcg_enc_frame* frames, uint32_t count, std::vector<EFrame>& ef)
{
    std::vector<EPlane> planes;
    std::vector<VSeg> segs;
    std::vector<VTile> tiles;
    std::vector<VPlaneD> vps;
    std::vector<EWork> work;
    std::vector<uint32_t> coded, tile_ids, ctile;
    std::vector<int32_t> lanes;
    std::vector<uint8_t> ext((size_t)count * V8_EXT, 0);
    ef.assign(count, EFrame());
    uint64_t pix_elems = 0, nblk = 0, ops_words = 0, stage_bytes = 0, pkt_bytes = 0;
    for (uint32_t f = 0; f < count; ++f) {
        const tcg_enc_frame& F = frames[f];
        ef[f].slice0 = (uint32_t)vps.size();
        ef[f].nslices = 3u;
        memset(ef[f].hdr, 0, sizeof(ef[f].hdr));
        memcpy(ef[f].hdr, F.header, 53);
        ext[(size_t)f * V8_EXT] = (uint8_t)F.v8_sb_log2;
        ext[(size_t)f * V8_EXT + 1u] = (uint8_t)F.v8_tile_log2;
        const uint32_t sb = 1u << F.v8_sb_log2;
        uint64_t fbound = 53u + V8_EXT;
        for (uint32_t p = 0; p < 3u; ++p) {
            const tcg_enc_plane& I = F.plane[p];
            EPlane P;
            memset(&P, 0, sizeof(P));
            P.pix_off = pix_elems;
            pix_elems = align_up(pix_elems + (uint64_t)I.vis_w * I.vis_h, 64);
            P.vis_w = I.vis_w; P.vis_h = I.vis_h; P.coded_w = I.coded_w; P.coded_h = I.coded_h;
            P.cols = I.cols; P.rows = I.rows; P.kind = TCG_PLANE_COLOR;
            P.bd = F.bit_depth;
            P.blk0 = (uint32_t)nblk;
            P.fclamp = I.fclamp;
            P.q_is_one = 1u;
            for (int i = 0; i < 64; ++i) {
                P.Q[i] = I.Q[i];
                if (I.Q[i] != 1u) { P.q_is_one = 0u; }
                div_magic(I.Q[i] != 0u ? I.Q[i] : 1u, &P.Qm[i], &P.Qsh[i]);
            }
            P.seg0 = (uint32_t)segs.size();
            P.sb_log2 = F.v8_sb_log2;
            const uint32_t pg = (uint32_t)planes.size();
            const uint32_t blocks = I.cols * I.rows;
            const uint32_t S = (blocks + sb - 1u) / sb;
            const uint32_t tr = F.v8_tile_log2 == 0u ? 0u : 1u << F.v8_tile_log2;
            const uint32_t T = (tr == 0u || I.rows == 0u) ? 1u : (I.rows + tr - 1u) / tr;
            VPlaneD D;
            memset(&D, 0, sizeof(D));
            D.seg0 = P.seg0; D.nseg = S; D.tile0 = (uint32_t)tiles.size(); D.ntile = T;
            const uint32_t vpi = (uint32_t)vps.size();
            for (uint32_t k = 0; k < S; ++k) {
                VSeg G;
                memset(&G, 0, sizeof(G));
                G.frame = f; G.plane = vpi; G.tile = 0xFFFFFFFFu;
                G.blk0 = P.blk0 + k * sb;
                G.nblk = std::min(sb, blocks - k * sb);
                G.sidx = k;
                G.qdb = I.qdb;
                G.op_base = ops_words;
                ops_words += (uint64_t)G.nblk * 256u + 256u;
                G.stage_cap = (uint64_t)G.nblk * 512u + 64u;
                G.stage_base = stage_bytes;
                stage_bytes = align_up(stage_bytes + G.stage_cap, 256);
                fbound += V8_DIR + 4u + G.stage_cap;
                segs.push_back(G);
            }
            for (uint32_t t = 0; t < T; ++t) {
                const uint64_t fb = tr == 0u ? 0u : (uint64_t)t * tr * I.cols;
                const uint64_t fn = tr == 0u ? (uint64_t)blocks : (uint64_t)(t + 1u) * tr * I.cols;
                uint32_t sf = (uint32_t)std::min<uint64_t>(fb / sb, S), sn = (uint32_t)std::min<uint64_t>(fn / sb, S);
                sn = std::max(sn, sf);
                VTile V;
                memset(&V, 0, sizeof(V));
                V.frame = f; V.plane = pg; V.tidx = t; V.seg0 = P.seg0 + sf; V.nseg = sn - sf;
                V.blk0 = P.blk0 + sf * sb;
                V.nblk = sn > sf ? std::min(sn * sb, blocks) - sf * sb : 0u;
                const uint32_t ti = (uint32_t)tiles.size();
                for (uint32_t k = sf; k < sn; ++k) {
                    segs[P.seg0 + k].tile = ti;
                    coded.push_back(P.seg0 + k);
                }
                for (uint32_t lb = 0; lb < V.nblk; lb += 256u) {
                    EWork w = {ti, lb, std::min(256u, V.nblk - lb), 0u};
                    work.push_back(w);
                }
                for (uint32_t k = sf; k < sn; k += 32u) {
                    ctile.push_back(ti);
                    for (uint32_t l = 0; l < 32u; ++l) { lanes.push_back(k + l < sn ? (int32_t)(P.seg0 + k + l) : -1); }
                }
                tile_ids.push_back(ti);
                tiles.push_back(V);
                fbound += V8_TABLE + 4u;
            }
            nblk += blocks;
            planes.push_back(P);
            vps.push_back(D);
        }
        ef[f].pkt_base = pkt_bytes;
        pkt_bytes = align_up(pkt_bytes + fbound, 256);
    }
    const uint32_t nseg = (uint32_t)segs.size(), nt = (uint32_t)tiles.size(), ncoded = (uint32_t)coded.size();
    const uint32_t nwarps = (uint32_t)ctile.size();
    const size_t desc_bytes = align_up(planes.size() * sizeof(EPlane), 256) + align_up(segs.size() * sizeof(VSeg), 256) +
                              align_up(tiles.size() * sizeof(VTile), 256) + align_up(vps.size() * sizeof(VPlaneD), 256) +
                              align_up(count * sizeof(EFrame), 256) + align_up(work.size() * sizeof(EWork) + 16, 256) +
                              align_up((planes.size() + coded.size() + tile_ids.size() + ctile.size()) * 4u + 16u, 256) +
                              align_up(lanes.size() * 4u + 16u, 256) + align_up(ext.size() + 16u, 256) +
                              align_up(planes.size() * 4u + 16u, 256) + 1024u;
    const size_t res_bytes = align_up((size_t)nseg * sizeof(VSegRes), 256) + align_up((size_t)nt * sizeof(ESliceRes), 256);
    if (!dreserve(C, B_PIX, pix_elems * 2u + 256) || !dreserve(C, B_COEF, nblk * 256u + 256) ||
        !dreserve(C, B_MASK, nblk * 8u + 256) || !dreserve(C, B_DCM, nblk * 4u + 256) ||
        !dreserve(C, B_NOPS, nblk * 4u + 256) || !dreserve(C, B_OPOFF, nblk * 4u + 256) ||
        !dreserve(C, B_UMAP, (nblk + 31u) / 32u * 4u + 256) ||
        !dreserve(C, B_HIST, (size_t)nt * H_BINS * 4u + 256) || !dreserve(C, B_STAB, (size_t)nt * T_SIZE * 4u + 256) ||
        !dreserve(C, B_TMP0, (size_t)nt * PREFIX_MAX + 256) || !dreserve(C, B_OPS, ops_words * 4u + 256) ||
        !dreserve(C, B_STAGE, stage_bytes + 256) || !dreserve(C, B_SRES, res_bytes + 256) ||
        !dreserve(C, B_FRES, (size_t)count * (sizeof(EFrameRes) + 4u) + 256) || !dreserve(C, B_PKT, pkt_bytes + 256) ||
        !dreserve(C, B_DESC, desc_bytes) || !hreserve(C, 0, desc_bytes) ||
        !hreserve(C, 1, (size_t)count * sizeof(EFrameRes) + 4096)) {
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
    std::vector<uint32_t> cplanes(planes.size());
    for (uint32_t i = 0; i < (uint32_t)planes.size(); ++i) { cplanes[i] = i; }
    const size_t o_pl = put(planes.data(), planes.size() * sizeof(EPlane));
    const size_t o_sg = put(segs.data(), segs.size() * sizeof(VSeg));
    const size_t o_tl = put(tiles.data(), tiles.size() * sizeof(VTile));
    const size_t o_vp = put(vps.data(), vps.size() * sizeof(VPlaneD));
    const size_t o_fr = put(ef.data(), count * sizeof(EFrame));
    const size_t o_wk = put(work.data(), work.size() * sizeof(EWork));
    const size_t o_cp = put(cplanes.data(), cplanes.size() * 4u);
    const size_t o_cd = put(coded.data(), coded.size() * 4u);
    const size_t o_ti = put(tile_ids.data(), tile_ids.size() * 4u);
    const size_t o_ct = put(ctile.data(), ctile.size() * 4u);
    const size_t o_ln = put(lanes.data(), lanes.size() * 4u);
    const size_t o_ex = put(ext.data(), ext.size());
    std::vector<uint32_t> pstart(planes.size());  // first block of each plane (unit lookup)
    for (size_t i = 0; i < planes.size(); ++i) { pstart[i] = planes[i].blk0; }
    const size_t o_ps = put(pstart.data(), pstart.size() * 4u);
    call_begin(C);
    TCG_CHECK(cudaMemcpyAsync(dd, hd, o, cudaMemcpyHostToDevice, st));
    const EPlane* d_pl = (const EPlane*)(dd + o_pl);
    const VSeg* d_sg = (const VSeg*)(dd + o_sg);
    VTile* d_tl = (VTile*)(dd + o_tl);
    VPlaneD* d_vp = (VPlaneD*)(dd + o_vp);
    const EFrame* d_fr = (const EFrame*)(dd + o_fr);
    const EWork* d_wk = (const EWork*)(dd + o_wk);
    const uint32_t* d_cp = (const uint32_t*)(dd + o_cp);
    const uint32_t* d_cd = (const uint32_t*)(dd + o_cd);
    const uint32_t* d_ti = (const uint32_t*)(dd + o_ti);
    const uint32_t* d_ct = (const uint32_t*)(dd + o_ct);
    const int32_t* d_ln = (const int32_t*)(dd + o_ln);
    const uint32_t* d_ps = (const uint32_t*)(dd + o_ps);
    const uint8_t* d_ex = dd + o_ex;
    uint16_t* d_pix = dptr<uint16_t>(C, B_PIX);
    for (uint32_t f = 0, pg = 0; f < count; ++f) {
        for (uint32_t p = 0; p < 3u; ++p, ++pg) {
            const tcg_enc_plane& I = frames[f].plane[p];
            if (I.stride == I.vis_w) {
                TCG_CHECK(cudaMemcpyAsync(d_pix + planes[pg].pix_off, I.src, (size_t)I.vis_w * I.vis_h * 2u,
                                          cudaMemcpyDefault, st));
            } else {
                TCG_CHECK(cudaMemcpy2DAsync(d_pix + planes[pg].pix_off, (size_t)I.vis_w * 2u, I.src, I.stride * 2u,
                                            (size_t)I.vis_w * 2u, I.vis_h, cudaMemcpyDefault, st));
            }
        }
    }
    TCG_CHECK(cudaEventRecord(C->gate, st));
    uint8_t* d_res = dptr<uint8_t>(C, B_SRES);
    VSegRes* d_sres = (VSegRes*)d_res;
    ESliceRes* d_tres = (ESliceRes*)(d_res + align_up((size_t)nseg * sizeof(VSegRes), 256));
    EFrameRes* d_fres = dptr<EFrameRes>(C, B_FRES);
    uint32_t* d_aerr = reinterpret_cast<uint32_t*>(dptr<uint8_t>(C, B_FRES) + align_up(count * sizeof(EFrameRes), 16));
    TCG_CHECK(cudaMemsetAsync(d_res, 0, res_bytes, st));
    TCG_CHECK(cudaMemsetAsync(d_aerr, 0, (size_t)count * 4u, st));
    TCG_CHECK(cudaMemsetAsync(dptr<uint32_t>(C, B_HIST), 0, (size_t)nt * H_BINS * 4u, st));
    const DevTables& Tb = tables();
    int32_t* d_coef = dptr<int32_t>(C, B_COEF);
    uint64_t* d_mask = dptr<uint64_t>(C, B_MASK);
    uint32_t* d_dcm = dptr<uint32_t>(C, B_DCM);
    uint32_t* d_nops = dptr<uint32_t>(C, B_NOPS);
    uint32_t* d_opoff = dptr<uint32_t>(C, B_OPOFF);
    uint32_t* d_hist = dptr<uint32_t>(C, B_HIST);
    uint32_t* d_stab = dptr<uint32_t>(C, B_STAB);
    uint8_t* d_prefix = dptr<uint8_t>(C, B_TMP0);
    uint32_t* d_ops = dptr<uint32_t>(C, B_OPS);
    uint8_t* d_stage = dptr<uint8_t>(C, B_STAGE);
    uint8_t* d_pkt = dptr<uint8_t>(C, B_PKT);
    bool any_wide = false;
    for (const EPlane& P : planes) { any_wide = any_wide || P.bd > 12u; }
    uint32_t* d_umap = dptr<uint32_t>(C, B_UMAP);
    TCG_LAUNCH(C, K_UNIT_MAP, k_unit_map, (uint32_t)((nblk + 8191u) / 8192u), 256, 0, d_ps, 1u,
               (uint32_t)planes.size(), (uint32_t)nblk, d_umap);
    TCG_LAUNCH(C, K_FDCT, k_fdct, (uint32_t)((nblk + FB_BLOCKS - 1u) / FB_BLOCKS), 256, 0, d_pl, d_cp,
               (uint32_t)planes.size(), (uint32_t)nblk, d_pix, d_coef, d_mask, d_ps, d_umap);
    if (any_wide) {
        TCG_LAUNCH(C, K_FDCT, k_fdct_wide, (uint32_t)((nblk + 127u) / 128u), 128, 0, d_pl, d_cp, (uint32_t)planes.size(),
                   (uint32_t)nblk, d_pix, d_coef, d_mask);
    }
    const size_t tok_smem = H_BINS * 32u * 4u;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_v8_tokens, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tok_smem);
        attr_set = true;
    }
    if (!work.empty()) {
        TCG_LAUNCH(C, K_TOKENS, k_v8_tokens, (uint32_t)work.size(), 256, tok_smem, d_wk, d_tl, d_pl, d_coef, d_mask,
                   d_dcm, d_nops, d_hist, d_tres);
    }
    TCG_LAUNCH(C, K_SELECT, k_select, nt, 32, 0, nullptr, d_ti, d_hist, Tb.log2, d_stab, d_prefix, d_tres);
    if (ncoded > 0u) {
        TCG_LAUNCH(C, K_OPSCAN, k_v8_opscan, (ncoded + 7u) / 8u, 256, 0, d_sg, d_cd, ncoded, d_nops, d_opoff, d_ops,
                   d_sres);
        TCG_LAUNCH(C, K_OPGEN, k_v8_opgen, dim3((uint32_t)work.size(), 32), 256, 0, d_wk, d_tl, d_pl, d_sg, d_coef,
                   d_mask, d_dcm, d_opoff, d_tres, d_ops);
        TCG_LAUNCH(C, K_CHAIN, k_v8_chain, nwarps, 32, V8CH_SMEM, d_sg, d_ln, d_ct, d_ops, d_stab, Tb.div_m, Tb.div_l,
                   d_stage, d_sres);
    }
    TCG_LAUNCH(C, K_PACK_SIZES, k_v8_sizes, count, 1024, 0, d_fr, d_vp, d_sg, d_sres, d_tl, d_tres, d_fres, d_pkt, d_ex);
    TCG_LAUNCH(C, K_PACK_COPY, k_v8_copy, (nseg + 7u) / 8u, 256, 0, d_fr, d_vp, d_sg, nseg, d_sres, d_stage, d_pkt);
    TCG_LAUNCH(C, K_PACK_CRC, k_v8_tiles, nt, 256, 0, d_fr, d_tl, d_tres, d_prefix, Tb.crc, d_pkt);
    TCG_LAUNCH(C, K_PACK_HEADER, k_pack_header, (count + 127u) / 128u, 128, 0, d_fr, count, d_fres, Tb.crc, d_pkt);
    TCG_CHECK(cudaGetLastError());
    EFrameRes* hf = (EFrameRes*)C->h[1].p;
    uint32_t* ha = (uint32_t*)((uint8_t*)C->h[1].p + align_up(count * sizeof(EFrameRes), 16));
    TCG_CHECK(cudaMemcpyAsync(hf, d_fres, count * sizeof(EFrameRes), cudaMemcpyDeviceToHost, st));
    TCG_CHECK(cudaMemcpyAsync(ha, d_aerr, count * 4u, cudaMemcpyDeviceToHost, st));
    return 0;
}

// Wait for a launched batch's per-frame results, fill res and enqueue the copy
// of every packet that fits its buffer (the caller synchronises the stream).
static int32_t encode_results(Ctx* C, const std::vector<EFrame>& ef, uint8_t* const* outs, const size_t* caps,
                              tcg_enc_result* res)
{
    const uint32_t count = (uint32_t)ef.size();
    cudaStream_t st = C->stream;
    const uint8_t* d_pkt = dptr<uint8_t>(C, B_PKT);
    const EFrameRes* hf = (const EFrameRes*)C->h[1].p;
    const uint32_t* ha = (const uint32_t*)((const uint8_t*)C->h[1].p + align_up(count * sizeof(EFrameRes), 16));
    TCG_CHECK(cudaStreamSynchronize(st));
    for (uint32_t f = 0; f < count; ++f) {
        tcg_enc_result& r = res[f];
        memset(&r, 0, sizeof(r));
        r.alpha_max_err = ha[f];
        if (hf[f].err != 0u) {
            r.rc = TCG_ERR_INVALID_ARGUMENT;
            continue;
        }
        if (hf[f].size == 0xFFFFFFFFu) {
            r.rc = TCG_ERR_LIMIT_EXCEEDED;
            continue;
        }
        r.packet_size = hf[f].size;
        r.color_payload = hf[f].color_payload;
        r.alpha_payload = hf[f].alpha_payload;
        r.color_slices = hf[f].color_slices;
        r.alpha_slices = hf[f].alpha_slices;
        if ((size_t)r.packet_size > caps[f]) {
            r.rc = TCG_ERR_BUFFER_TOO_SMALL;
            continue;
        }
        if (outs[f] != nullptr) {
            TCG_CHECK(cudaMemcpyAsync(outs[f], d_pkt + ef[f].pkt_base, r.packet_size, cudaMemcpyDefault, st));
        }
        r.rc = 0;
    }
    return 0;
}

static int32_t encode_impl(Ctx* C, const tcg_enc_frame* frames, uint32_t count, uint8_t* const* outs,
                           const size_t* caps, tcg_enc_result* res)
{
    std::vector<EFrame> ef;
    int32_t rc = count > 0u && frames[0].v8_sb_log2 != 0u ? encode_launch_v8(C, frames, count, ef)
                                                          : encode_launch(C, frames, count, nullptr, ef);
    if (rc == 0) { rc = encode_results(C, ef, outs, caps, res); }
    if (rc != 0) { return rc; }
    TCG_CHECK(cudaStreamSynchronize(C->stream));
    call_end(C);
    return 0;
}

// Host-memory batch in chunks on as many contexts (pipeline_plan): all chunks
// are launched first, chunk i's sample copies queued behind chunk i-1's, then
// each chunk's results are read and its packets copied back in order while
// later chunks still compute. The reported device time spans the first
// chunk's start to the last chunk's end.
static int32_t encode_pipelined(const tcg_enc_frame* frames, const uint32_t* starts, uint32_t k, uint8_t* const* outs,
                                const size_t* caps, tcg_enc_result* res)
{
    Ctx* cs[PIPE_MAX_CHUNKS] = {};
    std::vector<EFrame> ef[PIPE_MAX_CHUNKS];
    int32_t rc = 0;
    uint32_t launched = 0;
    for (uint32_t i = 0; i < k && rc == 0; ++i) {
        cs[i] = ctx_acquire();
        if (cs[i] == nullptr) {
            rc = TCG_ERR_NOT_IMPLEMENTED;
            break;
        }
        launched = i + 1u;
        rc = encode_launch(cs[i], frames + starts[i], starts[i + 1] - starts[i], i ? cs[i - 1]->gate : nullptr, ef[i]);
    }
    for (uint32_t i = 0; i < launched && rc == 0; ++i) {
        rc = encode_results(cs[i], ef[i], outs + starts[i], caps + starts[i], res + starts[i]);
    }
    double span = 0.0;
    for (uint32_t i = 0; i < launched; ++i) {
        const cudaError_t e = cudaStreamSynchronize(cs[i]->stream);
        if (rc == 0 && e != cudaSuccess) { rc = cuda_fail(e, "pipelined encode"); }
        if (rc == 0) {
            call_end(cs[i]);
            span = std::max(span, event_span_ms(cs[0]->t0, cs[i]->t1));
        }
    }
    for (uint32_t i = 0; i < launched; ++i) { ctx_release(cs[i]); }
    if (rc == 0) { set_last_ms(span); }
    return rc;
}

}  // namespace tcg

// ------------------------------------------------------------ sized sessions
//
// A session leases one context for the call. Host-memory sample planes are
// uploaded once into the context's grow-only B_SIZED_PIX buffer. Probe packets
// go to B_SIZED_PKT, split in two halves used in turn by successive launches,
// so the packets of the last two launches stay available; an older one is
// reported as no longer kept and the caller encodes that qp again.

struct tcg_sized {
    tcg::Ctx* C = nullptr;
    const void* src[4] = {};                     // plane sources the variants read
    size_t stride[4] = {};
    uint32_t launches = 0;                       // encode calls so far
    size_t half = 0;                             // bytes of one half of B_SIZED_PKT
    struct Slot { uint32_t launch; size_t off, cap; };
    std::vector<Slot> slot;
};

extern "C" int32_t tcg_sized_open(const tcg_enc_frame* base, tcg_sized** out)
{
    *out = nullptr;
    tcg::Ctx* C = tcg::ctx_acquire();
    if (C == nullptr) { return TCG_ERR_NOT_IMPLEMENTED; }
    tcg_sized* s = new tcg_sized();
    s->C = C;
    size_t host_bytes = 0;
    for (uint32_t p = 0; p < base->planes; ++p) {
        const tcg_enc_plane& I = base->plane[p];
        s->src[p] = I.src;
        s->stride[p] = I.stride;
        if (tcg::host_memory(I.src)) { host_bytes += tcg::align_up((size_t)I.vis_w * I.vis_h * 2u, 256); }
    }
    if (host_bytes > 0) {
        // every probe reads the samples from HBM: one upload, tight rows
        if (!tcg::dreserve(C, tcg::B_SIZED_PIX, host_bytes)) {
            tcg_sized_close(s);
            return TCG_ERR_OUT_OF_MEMORY;
        }
        size_t off = 0;
        for (uint32_t p = 0; p < base->planes; ++p) {
            const tcg_enc_plane& I = base->plane[p];
            if (!tcg::host_memory(I.src)) { continue; }
            uint8_t* dst = tcg::dptr<uint8_t>(C, tcg::B_SIZED_PIX) + off;
            const cudaError_t e = cudaMemcpy2DAsync(dst, (size_t)I.vis_w * 2u, I.src, I.stride * 2u,
                                                    (size_t)I.vis_w * 2u, I.vis_h, cudaMemcpyDefault, C->stream);
            if (e != cudaSuccess) {
                tcg_sized_close(s);
                return tcg::cuda_fail(e, "sized upload");
            }
            s->src[p] = dst;
            s->stride[p] = I.vis_w;
            off += tcg::align_up((size_t)I.vis_w * I.vis_h * 2u, 256);
        }
    }
    *out = s;
    return 0;
}

extern "C" int32_t tcg_sized_encode(tcg_sized* s, const tcg_enc_frame* frames, uint32_t count, const size_t* caps,
                                    tcg_enc_result* res, uint32_t* slots)
{
    if (count == 0u) { return 0; }
    std::vector<tcg_enc_frame> fr(frames, frames + count);
    std::vector<uint8_t*> outs(count);
    size_t need = 0;
    for (uint32_t i = 0; i < count; ++i) {
        for (uint32_t p = 0; p < fr[i].planes; ++p) {
            fr[i].plane[p].src = (const uint16_t*)s->src[p];
            fr[i].plane[p].stride = s->stride[p];
        }
        need += tcg::align_up(caps[i], 256);
    }
    if (need > s->half) {
        // growing the store drops what it kept
        s->half = need;
        for (auto& k : s->slot) { k.launch = UINT32_MAX; }
    }
    if (!tcg::dreserve(s->C, tcg::B_SIZED_PKT, 2u * s->half)) { return TCG_ERR_OUT_OF_MEMORY; }
    const uint32_t launch = s->launches++;
    size_t off = (launch & 1u) * s->half;
    uint8_t* base = tcg::dptr<uint8_t>(s->C, tcg::B_SIZED_PKT);
    for (uint32_t i = 0; i < count; ++i) {
        outs[i] = base + off;
        slots[i] = (uint32_t)s->slot.size();
        s->slot.push_back({launch, off, caps[i]});
        off += tcg::align_up(caps[i], 256);
    }
    return tcg::encode_impl(s->C, fr.data(), count, outs.data(), caps, res);
}

extern "C" int32_t tcg_sized_fetch(tcg_sized* s, uint32_t slot, uint8_t* out, size_t size)
{
    if (slot >= s->slot.size() || size > s->slot[slot].cap) {
        tcg_host_set_error(TCG_ERR_INVALID_ARGUMENT, "sized fetch: no such packet");
        return TCG_ERR_INVALID_ARGUMENT;
    }
    const tcg_sized::Slot& k = s->slot[slot];
    if (k.launch == UINT32_MAX || k.launch + 2u < s->launches) { return 1; }  // no longer kept
    if (size == 0u) { return 0; }
    TCG_CHECK(cudaMemcpyAsync(out, tcg::dptr<uint8_t>(s->C, tcg::B_SIZED_PKT) + k.off, size, cudaMemcpyDefault,
                              s->C->stream));
    TCG_CHECK(cudaStreamSynchronize(s->C->stream));
    return 0;
}

extern "C" void tcg_sized_close(tcg_sized* s)
{
    if (s == nullptr) { return; }
    cudaStreamSynchronize(s->C->stream);
    tcg::ctx_release(s->C);
    delete s;
}

extern "C" int32_t tcg_encode(const tcg_enc_frame* frames, uint32_t count, uint8_t* const* outs, const size_t* caps,
                              tcg_enc_result* res)
{
    uint32_t n8 = 0;
    for (uint32_t f = 0; f < count; ++f) { n8 += frames[f].v8_sb_log2 != 0u ? 1u : 0u; }
    if (n8 != 0u && n8 != count) {
        // V7-R2 and V8 frames run as two launch sequences, each in call order
        double ms = 0.0;
        for (int v8 = 0; v8 < 2; ++v8) {
            std::vector<tcg_enc_frame> fr;
            std::vector<uint8_t*> o;
            std::vector<size_t> c;
            std::vector<uint32_t> at;
            for (uint32_t f = 0; f < count; ++f) {
                if ((frames[f].v8_sb_log2 != 0u) != (v8 != 0)) { continue; }
                fr.push_back(frames[f]);
                o.push_back(outs[f]);
                c.push_back(caps[f]);
                at.push_back(f);
            }
            std::vector<tcg_enc_result> r(fr.size());
            const int32_t rc = tcg_encode(fr.data(), (uint32_t)fr.size(), o.data(), c.data(), r.data());
            if (rc != 0) { return rc; }
            ms += tcg_last_ms();
            for (size_t k = 0; k < at.size(); ++k) { res[at[k]] = r[k]; }
        }
        tcg::set_last_ms(ms);
        return 0;
    }
    if (count >= 2u && n8 == 0u && tcg::host_memory(frames[0].plane[0].src)) {
        std::vector<uint64_t> bytes(count, 0);
        for (uint32_t f = 0; f < count; ++f) {
            for (uint32_t p = 0; p < frames[f].planes; ++p) {
                bytes[f] += (uint64_t)frames[f].plane[p].vis_w * frames[f].plane[p].vis_h * 2u;
            }
        }
        uint32_t starts[tcg::PIPE_MAX_CHUNKS + 1];
        const uint32_t k = tcg::pipeline_plan(false, bytes.data(), count, starts);
        if (k > 1u) { return tcg::encode_pipelined(frames, starts, k, outs, caps, res); }
    }
    tcg::Ctx* c = tcg::ctx_acquire();
    if (c == nullptr) { return TCG_ERR_NOT_IMPLEMENTED; }
    const int32_t rc = tcg::encode_impl(c, frames, count, outs, caps, res);
    tcg::ctx_release(c);
    return rc;
}
