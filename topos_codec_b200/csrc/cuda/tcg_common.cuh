// tcg_common.cuh - device helpers shared by the encode and decode kernels:
// symbol maps, context buckets, rANS model normalisation, the exact 8x8
// integer transforms, CRC-32 (slicing-by-8 + GF(2) combination).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tcg {

// ------------------------------- constants -------------------------------

constexpr uint32_t RANS_L = 1u << 23;
constexpr uint32_t DC_SYMS = 29, RUN_SYMS = 64, LVL_SYMS = 28;
constexpr uint32_t POS_CTX = 4, PREV_CTX = 5, DCP_CTX = 5;
// histogram layout per colour slice (u32 counts)
constexpr uint32_t H_DC = 0;                                  // [29]
constexpr uint32_t H_RUN = H_DC + DC_SYMS;                    // [64]
constexpr uint32_t H_LVL = H_RUN + RUN_SYMS;                  // [28]
constexpr uint32_t H_JPOS = H_LVL + LVL_SYMS;                 // [4][28]
constexpr uint32_t H_JPREV = H_JPOS + POS_CTX * LVL_SYMS;     // [5][28]
constexpr uint32_t H_JDC = H_JPREV + PREV_CTX * LVL_SYMS;     // [5][29]
constexpr uint32_t H_BINS = H_JDC + DCP_CTX * DC_SYMS;        // 518
// per-slice coding table (u32 f<<12|cum): dc[5][29], run[64], lvl[5][28]
constexpr uint32_t T_DC = 0, T_RUN = 145, T_LVL = 209, T_SIZE = 349;
constexpr uint32_t PREFIX_MAX = 352;

__device__ __constant__ uint8_t c_zigzag[64] = {
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};
// the same order for compile-time indexing (unrolled loops over registers)
__device__ constexpr uint8_t k_zigzag[64] = {
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// ------------------------------- small maps -------------------------------

__device__ __forceinline__ uint32_t bitlen32(uint32_t m) { return 32u - (uint32_t)__clz(m); }

__device__ __forceinline__ uint32_t map_s(int32_t v)
{
    return v >= 0 ? (uint32_t)v << 1 : (((uint32_t)(-(int64_t)v)) << 1) - 1u;
}

__device__ __forceinline__ int32_t unmap_s(uint32_t m)
{
    return (m & 1u) == 0u ? (int32_t)(m >> 1) : -(int32_t)((m >> 1) + 1u);
}

__device__ __forceinline__ int32_t dc_pred(bool hl, int32_t l, bool ht, int32_t t)
{
    if (hl && ht) {
        const int64_t s = (int64_t)l + t;
        return s >= 0 ? (int32_t)((s + 1) >> 1) : -(int32_t)((-s) >> 1);
    }
    return hl ? l : (ht ? t : 0);
}

__device__ __forceinline__ uint32_t pos_ctx(uint32_t pos) { return pos < 8u ? 0u : pos < 16u ? 1u : pos < 32u ? 2u : 3u; }
__device__ __forceinline__ uint32_t cat_bucket(uint32_t c) { return c == 0u ? 0u : c == 1u ? 1u : c <= 3u ? 2u : 3u; }
__device__ __forceinline__ uint32_t prev_ctx(uint32_t cat, bool has) { return has ? cat_bucket(cat) : 4u; }
__device__ __forceinline__ uint32_t dcp_ctx(uint32_t cat, bool has) { return has ? 1u + cat_bucket(cat) : 0u; }

// number of raw chunks carrying a category suffix (cat-1 bits, split above 23)
__device__ __forceinline__ uint32_t suffix_chunks(uint32_t cat) { return cat <= 1u ? 0u : (cat - 1u > 23u ? 2u : 1u); }

// ------------------------------- rANS models -------------------------------

// Proportional 8-bit row bytes; an all-zero row becomes {1,0,...}.
__device__ inline void row_encode(uint8_t* out, uint32_t nsym, const uint32_t* cnt)
{
    uint64_t total = 0;
    for (uint32_t s = 0; s < nsym; ++s) { total += cnt[s]; }
    if (total == 0u) {
        for (uint32_t s = 0; s < nsym; ++s) { out[s] = s == 0u ? 1u : 0u; }
        return;
    }
    for (uint32_t s = 0; s < nsym; ++s) {
        if (cnt[s] == 0u) { out[s] = 0u; continue; }
        uint64_t v = ((uint64_t)cnt[s] * 255u + total / 2u) / total;
        out[s] = (uint8_t)(v == 0u ? 1u : (v > 255u ? 255u : v));
    }
}

// Deterministic normalisation of byte counts to a 4096 total: floor share
// with a floor of 1 for used symbols, then -1 from the largest frequency
// (lowest index on ties) or +1 to the largest remainder (lowest index on
// ties). Returns false for an all-zero row.
__device__ inline bool model_from_bytes(const uint8_t* b, uint32_t nsym, uint16_t* freq, uint16_t* cum)
{
    uint32_t total = 0;
    for (uint32_t s = 0; s < nsym; ++s) { total += b[s]; }
    if (total == 0u) { return false; }
    uint32_t f[64], rem[64], sum = 0;
    for (uint32_t s = 0; s < nsym; ++s) {
        const uint32_t sc = (uint32_t)b[s] * 4096u;
        f[s] = b[s] == 0u ? 0u : sc / total;
        rem[s] = sc % total;
        if (b[s] != 0u && f[s] == 0u) { f[s] = 1u; }
        sum += f[s];
    }
    while (sum > 4096u) {
        int big = -1;
        for (uint32_t s = 0; s < nsym; ++s) {
            if (f[s] > 1u && (big < 0 || f[s] > f[big])) { big = (int)s; }
        }
        if (big < 0) { break; }
        f[big]--; rem[big] = 0u; sum--;
    }
    while (sum < 4096u) {
        int best = -1;
        for (uint32_t s = 0; s < nsym; ++s) {
            if (b[s] == 0u) { continue; }
            if (best < 0 || rem[s] > rem[best]) { best = (int)s; }
        }
        if (best < 0) { break; }
        f[best]++; rem[best] = 0u; sum++;
    }
    if (sum != 4096u) { return false; }
    uint32_t acc = 0;
    for (uint32_t s = 0; s < nsym; ++s) {
        freq[s] = (uint16_t)f[s];
        cum[s] = (uint16_t)acc;
        acc += f[s];
    }
    return true;
}

// ---------------------------- integer transforms ----------------------------
// Basis M[u][x] (|M| <= 13); even rows symmetric, odd rows antisymmetric, so
// each 8-point pass splits into sums and differences (exact integer regrouping).

#define TCG_M(u, k) ((int32_t)c_tm[(u) * 8 + (k)])
__device__ __constant__ int8_t c_tm[64] = {
    13, 13, 13, 13, 13, 13, 13, 13, 13, 11, 7, 1, -1, -7, -11, -13,
    12, 5, -5, -12, -12, -5, 5, 12, 11, -4, -13, -8, 8, 13, 4, -11,
    9, -9, -9, 9, 9, -9, -9, 9, 8, -13, 4, 11, -11, -4, 13, -8,
    5, -12, 12, -5, -5, 12, -12, 5, 1, -7, 11, -13, 13, -11, 7, -1};
__device__ __constant__ int32_t c_tw[64] = {
    2350, 4672, 4699, 4293, 4902, 4293, 4699, 4672,
    4672, 9288, 9343, 8535, 9747, 8535, 9343, 9288,
    4699, 9343, 9399, 8586, 9805, 8586, 9399, 9343,
    4293, 8535, 8586, 7843, 8957, 7843, 8586, 8535,
    4902, 9747, 9805, 8957, 10228, 8957, 9805, 9747,
    4293, 8535, 8586, 7843, 8957, 7843, 8586, 8535,
    4699, 9343, 9399, 8586, 9805, 8586, 9399, 9343,
    4672, 9288, 9343, 8535, 9747, 8535, 9343, 9288};
__device__ __constant__ int32_t c_te[8] = {1352, 680, 676, 740, 648, 740, 676, 680};

// 8-point forward pass on one line: out[v] = sum_k in[k] * M[v][k].
template <typename T>
__device__ __forceinline__ void fwd8(const T* in, T* out)
{
    T s[4], d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) { s[k] = in[k] + in[7 - k]; d[k] = in[k] - in[7 - k]; }
#pragma unroll
    for (int v = 0; v < 8; v += 2) {
        T e = 0, o = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) { e += s[k] * (T)TCG_M(v, k); o += d[k] * (T)TCG_M(v + 1, k); }
        out[v] = e;
        out[v + 1] = o;
    }
}

// F = M * x * M^T for 32-bit inputs (bit depth <= 12: |x| <= 2048, |F| < 2^25).
__device__ __forceinline__ void fdct8x8_i32(int32_t x[64], int32_t F[64])
{
    int32_t A[64];
#pragma unroll
    for (int y = 0; y < 8; ++y) { fwd8<int32_t>(x + y * 8, A + y * 8); }
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        int32_t col[8], out[8];
#pragma unroll
        for (int y = 0; y < 8; ++y) { col[y] = A[y * 8 + v]; }
        fwd8<int32_t>(col, out);
#pragma unroll
        for (int u = 0; u < 8; ++u) { F[u * 8 + v] = out[u]; }
    }
}

// Wide-sample forward transform (bit depth > 12): 64-bit accumulation, the
// second pass truncated to 32 bits, then the per-coefficient predistortion
// F' = round(F * 2^32 / (W * Eu * Ev)) with sign-split rounding.
__device__ inline void fdct8x8_wide(const int32_t x[64], int32_t F[64])
{
    int64_t A[64];
    for (int y = 0; y < 8; ++y) {
        int64_t in[8], out[8];
        for (int k = 0; k < 8; ++k) { in[k] = x[y * 8 + k]; }
        fwd8<int64_t>(in, out);
        for (int v = 0; v < 8; ++v) { A[y * 8 + v] = out[v]; }
    }
    for (int v = 0; v < 8; ++v) {
        int64_t col[8], out[8];
        for (int y = 0; y < 8; ++y) { col[y] = A[y * 8 + v]; }
        fwd8<int64_t>(col, out);
        for (int u = 0; u < 8; ++u) { F[u * 8 + v] = (int32_t)out[u]; }
    }
    for (int i = 0; i < 64; ++i) {
        const int64_t w = (int64_t)c_tw[i] * ((int64_t)c_te[i >> 3] * c_te[i & 7]);
        const int64_t num = (int64_t)F[i] * ((int64_t)1 << 32);
        F[i] = num >= 0 ? (int32_t)((2 * num + w) / (2 * w)) : -(int32_t)((-2 * num + w) / (2 * w));
    }
}

__device__ __forceinline__ int32_t round_shift32(int64_t v)
{
    return v >= 0 ? (int32_t)((v + ((int64_t)1 << 31)) >> 32) : -(int32_t)((-v + ((int64_t)1 << 31)) >> 32);
}

// Inverse: G = c (.) W, B = G * M, xhat = round(M^T * B / 2^32). Coefficients
// are clamped to +-2^30 first (callers already applied the bit-depth clamp).
__device__ inline void idct8x8(const int32_t c[64], int32_t xh[64])
{
    int64_t B[64];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        int64_t g[8];
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            int32_t t = c[u * 8 + v];
            t = t > (1 << 30) ? (1 << 30) : (t < -(1 << 30) ? -(1 << 30) : t);
            g[v] = (int64_t)t * c_tw[u * 8 + v];
        }
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            int64_t pe = 0, po = 0;
#pragma unroll
            for (int v = 0; v < 8; v += 2) { pe += g[v] * TCG_M(v, x); po += g[v + 1] * TCG_M(v + 1, x); }
            B[u * 8 + x] = pe + po;
            B[u * 8 + 7 - x] = pe - po;
        }
    }
#pragma unroll
    for (int x = 0; x < 8; ++x) {
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            int64_t qe = 0, qo = 0;
#pragma unroll
            for (int u = 0; u < 8; u += 2) { qe += (int64_t)TCG_M(u, y) * B[u * 8 + x]; qo += (int64_t)TCG_M(u + 1, y) * B[(u + 1) * 8 + x]; }
            xh[y * 8 + x] = round_shift32(qe + qo);
            xh[(7 - y) * 8 + x] = round_shift32(qe - qo);
        }
    }
}

// ------------------------------- unit lookup --------------------------------
// Kernels that take 32 blocks per CTA find each block's unit (plane or slice)
// from map[CTA], the unit holding the CTA's first block, and a short forward
// step over the units' first blocks: units are in increasing order of their
// first block and the first starts at block 0. k_unit_map fills map with one
// thread per 32-block chunk, each a binary search over the units' first blocks
// (unit i's first block at starts[i * stride]).
static __global__ void k_unit_map(const uint32_t* __restrict__ starts, uint32_t stride, uint32_t n, uint32_t total,
                                  uint32_t* __restrict__ map)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if ((uint64_t)c * 32u >= total) { return; }
    const uint32_t gb = c * 32u;
    uint32_t lo = 0, hi = n - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (starts[(size_t)mid * stride] <= gb) { lo = mid; } else { hi = mid - 1u; }
    }
    map[c] = lo;
}

__device__ __forceinline__ uint32_t unit_of(const uint32_t* __restrict__ starts, uint32_t stride, uint32_t n,
                                            uint32_t i, uint32_t gb)
{
    while (i + 1u < n && starts[(size_t)(i + 1u) * stride] <= gb) { ++i; }
    return i;
}

// ---------------------------------- CRC-32 ----------------------------------

// Multiply two polynomials modulo the CRC-32 polynomial (reflected bit order:
// bit 31 is the x^0 coefficient).
__device__ __forceinline__ uint32_t gf2_mulmod(uint32_t a, uint32_t b)
{
    uint32_t p = 0;
    for (int i = 0; i < 32; ++i) {
        if (a & 0x80000000u) { p ^= b; }
        a <<= 1;
        b = (b & 1u) ? (b >> 1) ^ 0xEDB88320u : b >> 1;
    }
    return p;
}

// x^(8 * nbytes) mod P, by repeated squaring of x^(2^k).
__device__ inline uint32_t gf2_xpow8n(uint64_t nbytes)
{
    uint32_t p = 0x80000000u;   // 1
    uint32_t sq = 0x00800000u;  // x^8
    while (nbytes != 0u) {
        if (nbytes & 1u) { p = gf2_mulmod(sq, p); }
        sq = gf2_mulmod(sq, sq);
        nbytes >>= 1;
    }
    return p;
}

// CRC of A||B from crc(A), crc(B) and the operator x^(8|B|) mod P.
__device__ __forceinline__ uint32_t crc_combine(uint32_t ca, uint32_t cb, uint32_t op_b)
{
    return gf2_mulmod(op_b, ca) ^ cb;
}

// Plain CRC-32 (init ~0, final ~0) of a byte range using slicing-by-8 tables
// t[8][256] (normally in shared memory).
__device__ inline uint32_t crc32_range(const uint8_t* p, uint64_t n, const uint32_t* t)
{
    uint32_t c = 0xFFFFFFFFu;
    while (n > 0u && ((uintptr_t)p & 7u) != 0u) { c = t[(c ^ *p++) & 0xFFu] ^ (c >> 8); --n; }
    const uint2* q = reinterpret_cast<const uint2*>(p);
    while (n >= 8u) {
        const uint2 w = __ldg(q++);
        const uint32_t a = c ^ w.x, b = w.y;
        c = t[7 * 256 + (a & 0xFFu)] ^ t[6 * 256 + ((a >> 8) & 0xFFu)] ^ t[5 * 256 + ((a >> 16) & 0xFFu)] ^
            t[4 * 256 + (a >> 24)] ^ t[3 * 256 + (b & 0xFFu)] ^ t[2 * 256 + ((b >> 8) & 0xFFu)] ^
            t[1 * 256 + ((b >> 16) & 0xFFu)] ^ t[b >> 24];
        n -= 8u;
    }
    p = reinterpret_cast<const uint8_t*>(q);
    while (n-- > 0u) { c = t[(c ^ *p++) & 0xFFu] ^ (c >> 8); }
    return c ^ 0xFFFFFFFFu;
}

// Block-cooperative CRC-32 of one byte range: every thread hashes whole
// chunks, then a binary tree combines neighbours. Needs blockDim.x threads,
// shared tables t (8 KB) and scratch of blockDim.x * 2 u32. Result valid in
// thread 0.
__device__ inline uint32_t crc32_block(const uint8_t* p, uint64_t n, const uint32_t* t, uint32_t* scratch)
{
    const uint32_t nt = blockDim.x, tid = threadIdx.x;
    uint64_t chunk = (n + nt - 1u) / nt;
    chunk = (chunk + 7u) & ~(uint64_t)7u;
    if (chunk < 64u) { chunk = 64u; }
    const uint64_t beg = (uint64_t)tid * chunk;
    const uint64_t len = beg >= n ? 0u : (n - beg < chunk ? n - beg : chunk);
    uint32_t* crc = scratch;
    uint32_t* lens = scratch + nt;
    crc[tid] = len == 0u ? 0u : crc32_range(p + beg, len, t);
    lens[tid] = (uint32_t)len;
    __syncthreads();
    for (uint32_t step = 1; step < nt; step <<= 1) {
        if ((tid % (2u * step)) == 0u && tid + step < nt) {
            const uint32_t lb = lens[tid + step];
            if (lb != 0u) {
                crc[tid] = lens[tid] == 0u ? crc[tid + step] : crc_combine(crc[tid], crc[tid + step], gf2_xpow8n(lb));
                lens[tid] += lb;
            }
        }
        __syncthreads();
    }
    return crc[0];
}

}  // namespace tcg
