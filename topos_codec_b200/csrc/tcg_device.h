/* tcg_device.h - internal C ABI between the C11 host library and the CUDA layer.
 *
 * The host library validates configurations, parses packet structure and
 * plans slices; it hands the CUDA layer fully resolved job descriptors made of
 * plain integers and pointers. The CUDA layer owns device memory, streams and
 * kernels, and returns per-frame results. Nothing here is public API.
 */
#ifndef TCG_DEVICE_H
#define TCG_DEVICE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* --------------------------------- encode --------------------------------- */

enum { TCG_PLANE_COLOR = 0, TCG_PLANE_ALPHA = 1 };

typedef struct tcg_enc_plane {
    const uint16_t* src;    /* caller samples (host or device memory), visible area */
    size_t stride;          /* uint16 elements between rows */
    uint32_t vis_w, vis_h;  /* visible plane size */
    uint32_t coded_w, coded_h;
    uint32_t cols, rows;    /* 8x8 blocks */
    uint32_t kind;          /* TCG_PLANE_COLOR / TCG_PLANE_ALPHA */
    uint32_t alpha_shift;   /* near-lossless alpha: 16 - alpha_bit_depth, else 0 */
    uint32_t qdb;           /* slice-header qp_delta_biased for this plane */
    uint32_t Q[64];         /* colour: quantiser steps, natural order */
    int64_t fclamp;         /* colour: coefficient clamp */
} tcg_enc_plane;

typedef struct tcg_enc_frame {
    uint32_t planes;
    uint32_t bit_depth;
    uint32_t slice_rows;
    uint32_t slices;        /* total slices (all planes) */
    tcg_enc_plane plane[4];
    uint8_t header[53];     /* frame header; packet size and header CRC are patched on the device */
    /* V8 segmented rANS: 0 for a V7-R2 frame, else the segment size log2
     * (3..5: 8/16/32 blocks per independent rANS chain) */
    uint32_t v8_sb_log2;
    uint32_t v8_tile_log2;  /* V8 tile height log2 in block rows (4..6), 0 = the whole plane */
} tcg_enc_frame;

typedef struct tcg_enc_result {
    int32_t rc;             /* TC_OK or the frame's error status */
    uint32_t packet_size;
    uint32_t color_payload, alpha_payload;
    uint32_t color_slices, alpha_slices;
    uint32_t alpha_max_err;
    uint32_t v8;            /* host side: the frame is V8 */
} tcg_enc_result;

/* Encodes count frames in one device launch sequence. For each frame whose
 * packet fits caps[i], the packet is copied to outs[i] (host or device memory).
 * Returns TC_OK when the device work ran (per-frame status in res[i].rc), or a
 * call-level error (out of device memory, CUDA failure). */
int32_t tcg_encode(const tcg_enc_frame* frames, uint32_t count,
                   uint8_t* const* outs, const size_t* caps, tcg_enc_result* res);

/* --------------------------------- decode --------------------------------- */

typedef struct tcg_dec_slice {
    uint32_t off;           /* payload offset within the packet */
    uint32_t size;          /* payload bytes */
    uint32_t crc;           /* slice-header CRC-32 of the payload */
    uint16_t plane, y0, bh;
    uint16_t qp;            /* effective qp of the slice */
    uint16_t k1, k2;        /* alpha Rice parameters */
} tcg_dec_slice;

typedef struct tcg_dec_frame {
    const uint8_t* packet;  /* host or device memory */
    size_t size;
    uint32_t planes, bit_depth, alpha_mode, alpha_shift;
    uint32_t vis_w[4], vis_h[4], coded_w[4], cols[4], rows[4];
    uint16_t qm[4][64];     /* per-plane quantisation matrix (natural order) */
    uint32_t refined;       /* refined qp scale table (header flags bit 3) */
    uint32_t deblock;       /* header flags bit 2 */
    uint32_t qp_base;
    uint32_t slices;
    const tcg_dec_slice* slice;
    uint16_t* dst[4];       /* caller planes (host or device memory) */
    size_t dst_stride[4];   /* uint16 elements */
    uint8_t* slice_status;  /* out: TC_FRAME_SLICE_* per slice (host memory) */
    int32_t skip;           /* in: nonzero = frame already rejected by the host */
    /* delivery (reference codec.c:8560-8640 slice tasks, 8700-8745 deblock):
     * planes >= `planes` are not decoded (their slices report OK, unchecked);
     * coefficients past zigzag position climit are dropped before the inverse
     * transform (63 keeps all); with `scaled`, plane p is delivered as
     * dst_w[p] x dst_h[p] samples, target (x, y) taking the reconstruction at
     * (x * vis_w / dst_w, y * vis_h / dst_h) rounded down; db_unit is the
     * grid of the delivered colour planes' deblocking (8 full size, 4 for an
     * exact half, 0 none) */
    uint32_t climit;
    uint32_t scaled;
    uint32_t dst_w[4], dst_h[4];
    uint32_t db_unit;
} tcg_dec_frame;

/* Size-targeted encode sessions. A session leases one context for its whole
 * life, holds a device copy of the frame's sample planes (uploaded once when
 * they are in host memory) and keeps the packets of its last two probe
 * launches on the device. tcg_sized_encode codes count variants of the
 * session's frame (the planes of `base` are used, whatever frames[i] holds;
 * headers and quantisers differ) in one launch sequence, with res[i] as from
 * tcg_encode and slots[i] naming the packet; caps[i] bounds packet i.
 * tcg_sized_fetch copies the first size bytes of a packet to out (host or
 * device memory): 0 when done, 1 when the packet is no longer kept (encode
 * that variant again), a negative status on error. */
typedef struct tcg_sized tcg_sized;
int32_t tcg_sized_open(const tcg_enc_frame* base, tcg_sized** out);
int32_t tcg_sized_encode(tcg_sized* s, const tcg_enc_frame* frames, uint32_t count, const size_t* caps,
                         tcg_enc_result* res, uint32_t* slots);
int32_t tcg_sized_fetch(tcg_sized* s, uint32_t slot, uint8_t* out, size_t size);
void tcg_sized_close(tcg_sized* s);

/* Decodes count frames in one device launch sequence; per-slice status is
 * written to each frame's slice_status. Returns TC_OK when the device work ran,
 * or a call-level error. */
int32_t tcg_decode(const tcg_dec_frame* frames, uint32_t count);

/* ---------------------------------- device --------------------------------- */

int32_t tcg_init(int32_t device);
void tcg_shutdown(void);
/* number of kernel launches issued by this process (all streams) */
uint64_t tcg_launch_count(void);
/* device time (ms, CUDA events on the library stream) of this thread's last call */
double tcg_last_ms(void);
/* split of a host-memory batch into pipelined chunks (see tcg_pipeline_plan) */
uint32_t tcg_pipeline_chunks(int32_t decode, const uint64_t* frame_bytes, uint32_t count, uint32_t* starts);
/* optional per-kernel event timing (process totals) */
void tcg_prof_enable(int32_t on);
void tcg_prof_reset(void);
int32_t tcg_prof_read(uint32_t id, const char** name, double* ms, uint64_t* launches);
/* nonzero when p is device (or managed) memory */
int32_t tcg_is_device_ptr(const void* p);
/* n bytes of device memory at src into host memory at dst (synchronous) */
int32_t tcg_read_device(void* dst, const void* src, size_t n);
/* free and total device memory of the library's device (0 and 0 without one) */
void tcg_mem_info(uint64_t* free_bytes, uint64_t* total_bytes);
/* gives back the device buffers idle call contexts keep from earlier calls */
void tcg_trim_idle(void);
/* the calling thread's lease class (-1: none): calls on a thread of class k
 * reuse idle call contexts last used by class k, or unused ones */
void tcg_set_lease_class(int32_t cls);
/* maps bytes of device memory into the library's memory pool ahead of use
 * (allocated and freed at once; the pool keeps it), so that calls that grow
 * their buffers later take it from the pool instead of mapping new memory */
int32_t tcg_pool_reserve(uint64_t bytes);

/* Structural walk of packets that live in device memory: per packet a record of
 * TCG_WALK_REC bytes = [64: packet bytes 0..60, zero beyond the packet]
 * [u32 slice headers walked][u32 end offset][8 pad][512 x 17-byte slice
 * headers], written to host_out. The walk stops exactly where a host parse of
 * the same bytes would run out of packet. */
#define TCG_WALK_REC (80u + 512u * 17u)
int32_t tcg_walk_packets(const uint8_t* const* pkts, const size_t* sizes, uint32_t n, uint8_t* host_out);

/* identical to the public definition in topos_codec.h */
#define TCG_NOALLOC_MAX_PACKETS 64u

/* The same walk for at most TCG_NOALLOC_MAX_PACKETS packets, with its tables
 * and records in the library's static device scratch instead of allocated
 * buffers (nothing is allocated). tcg_walk_record_noalloc copies record i of
 * the last walk on the current device to host_rec (TCG_WALK_REC bytes). */
int32_t tcg_walk_packets_noalloc(const uint8_t* const* pkts, const size_t* sizes, uint32_t n);
int32_t tcg_walk_record_noalloc(uint32_t i, uint8_t* host_rec);

/* ------------------------------- V8 decode ------------------------------- */

/* One V8 frame (segmented multi-chain rANS): the host has scanned the
 * structure and checked the tile tables; the device checks the tile CRCs,
 * decodes every segment whose tile matched, reconstructs all blocks (a segment
 * that is not decoded, or fails, reconstructs from zero coefficients: the mid
 * level) and writes the three colour planes. */
typedef struct tcg_v8_seg {
    uint32_t plane, blk0, nblk, tile;   /* blk0: first block within the plane */
    uint32_t off, len;                  /* stream bytes from the packet start */
    uint32_t qidx, pad;                 /* quantiser steps: q[qidx * 64 ..] */
} tcg_v8_seg;

typedef struct tcg_v8_tile {
    uint32_t plane, seg0, nseg, table_off;
    uint32_t stream_off, stream_bytes, crc, pad;
} tcg_v8_tile;

typedef struct tcg_v8_job {
    const uint8_t* packet;              /* host or device memory */
    size_t size;
    uint32_t bit_depth, sb_log2;
    uint32_t vis_w[3], vis_h[3], cols[3], rows[3];
    uint16_t* dst[3];                   /* host or device memory */
    size_t dst_stride[3];               /* uint16 elements */
    uint32_t nseg, ntile, nq;
    const tcg_v8_seg* seg;              /* plane-major, segment order */
    const tcg_v8_tile* tile;
    const uint32_t* q;                  /* nq x 64 steps, natural order */
    uint8_t* seg_fail;                  /* out, per segment: decode failed */
    uint8_t* tile_ok;                   /* out, per tile: CRC matched */
} tcg_v8_job;

/* count frames in one launch sequence */
int32_t tcg_decode_v8(const tcg_v8_job* jobs, uint32_t count);

/* provided by the host library: thread-local error detail */
void tcg_host_set_error(int32_t status, const char* text);
/* provided by the host library: exact log2 table (4097 doubles, index = freq) */
const double* tc_log2_table(void);

#ifdef __cplusplus
}
#endif

#endif /* TCG_DEVICE_H */
