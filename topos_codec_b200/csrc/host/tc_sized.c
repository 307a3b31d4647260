/* tc_sized.c - size-targeted encode (tc_frame_encode_sized).
 *
 * The reference searches qp one probe at a time: each probe is an exact
 * packet-size count at one qp, and the next qp depends on the sizes seen so
 * far (reference: native/src/codec/codec.c:7789-7880 entry, :7199-7262 legacy
 * linear search, :7271-7402 probe bookkeeping, :7404-7552 "r6" fast search,
 * :7554-7787 strict search). Its answer and every error it returns depend
 * only on those sizes, so this file runs the same three searches, step for
 * step, over a table of exact packet sizes that the GPU fills a window of qps
 * at a time: a probe of a qp the table lacks encodes it together with the
 * nearest unprobed qps (one batched launch sequence, the samples uploaded
 * once per call), and the packets of the last two launches stay on the
 * device, so the chosen one is normally copied out without a final encode.
 *
 * Process state as in the reference: the search mode (TOPOS_SIZED_SEARCH =
 * strict | linear | r6, or tc_dev_set_sized_mode), and the strict search's
 * cross-call qp hint (the last two distinct chosen qps with their sizes),
 * held by one process-wide record that a call borrows when it is free and
 * replaces by an empty one when another call holds it (reference:
 * codec.c:1002-1046, enc_loan_acquire). The hint only moves the first probe;
 * with sizes that fall as qp rises the chosen qp does not depend on it.
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/topos_codec_compat.h"
#include "../tcg_device.h"
#include "tc_internal.h"

#define SIZED_MAX_PTS 24
#define SIZED_PROBE_BUDGET 24u
/* the reference's exact-count probe needs a cache of every colour
 * coefficient; past 512 MiB of it (codec.c:6034) the strict search falls back
 * to the linear one */
#define SIZED_FCACHE_MAX_BYTES (512ull * 1024ull * 1024ull)
/* probe window: qps encoded per launch, and the device bytes one window may take */
#define SIZED_WINDOW 17u
#define SIZED_WINDOW_BYTES (24ull << 30)
/* batch form: searches side by side, and the device bytes all their windows may take */
#define SIZED_BATCH_WORKERS 6u
#define SIZED_BATCH_BYTES (96ull << 30)

/* ------------------------------------------------------------ process state */

typedef struct sized_hint {
    int valid;
    uint32_t q, bytes;         /* last chosen qp and its size */
    uint32_t prev, prev_bytes; /* the distinct one before it (bytes 0 = none) */
} sized_hint;

static sized_hint g_hint;
static atomic_int g_hint_busy;
static atomic_int g_mode;          /* 0 strict, 1 linear, 2 r6 */
static atomic_int g_mode_env_read;
static atomic_int g_hint_disable;
static atomic_int g_hint_model_disable;
static atomic_int g_m7_disable;
static _Atomic uint64_t g_iters;
static _Atomic uint64_t g_calls;

static void mode_env_init(void)
{
    if (atomic_exchange(&g_mode_env_read, 1) != 0) { return; }
    const char* env = getenv("TOPOS_SIZED_SEARCH");
    if (env == NULL) { return; }
    if (strcmp(env, "linear") == 0) {
        atomic_store(&g_mode, 1);
    } else if (strcmp(env, "r6") == 0) {
        atomic_store(&g_mode, 2);
    } else if (strcmp(env, "strict") == 0) {
        atomic_store(&g_mode, 0);
    }
}

/* reference: codec.c:7136-7143 */
TC_EXPORT void tc_dev_set_sized_mode(int32_t mode)
{
    atomic_store(&g_mode_env_read, 1);
    atomic_store(&g_mode, (mode < 0 || mode > 2) ? 0 : mode);
}

/* reference: codec.c:7147-7150 */
TC_EXPORT void tc_dev_set_sized_search(int legacy) { tc_dev_set_sized_mode(legacy ? 1 : 0); }
/* reference: codec.c:7155-7159 */
TC_EXPORT void tc_dev_set_qp_hint(int disable) { atomic_store(&g_hint_disable, disable ? 1 : 0); }
/* reference: codec.c:7165-7169 */
TC_EXPORT void tc_dev_set_qp_hint_model(int disable) { atomic_store(&g_hint_model_disable, disable ? 1 : 0); }
/* reference: codec.c:7174-7178 */
TC_EXPORT void tc_dev_set_sized_m7(int disable) { atomic_store(&g_m7_disable, disable ? 1 : 0); }

/* reference: codec.c:7110-7123 */
TC_EXPORT void tc_dev_sized_reset(void)
{
    atomic_store(&g_iters, 0u);
    atomic_store(&g_calls, 0u);
}
TC_EXPORT uint64_t tc_dev_sized_iters(void) { return atomic_load(&g_iters); }
TC_EXPORT uint64_t tc_dev_sized_calls(void) { return atomic_load(&g_calls); }

static void count_encode(void) { atomic_fetch_add(&g_iters, 1u); }

/* qps per probe launch for a frame with the given packet bound, samples and
 * colour blocks: device bytes of one probe are the packet, the samples and the
 * coder's per-block buffers */
static uint32_t sized_window(size_t cap, uint64_t samples, uint64_t cblocks)
{
    const uint64_t per = (uint64_t)cap + samples * 2u + cblocks * 2048u;
    uint64_t w = SIZED_WINDOW_BYTES / (per > 0u ? per : 1u);
    w = w < 1u ? 1u : (w > SIZED_WINDOW ? SIZED_WINDOW : w);
    return (uint32_t)w;
}

/* --------------------------------------------------------------- size table */

typedef struct size_table {
    tcg_sized* sess;
    const topos_frame_config* cfg;
    const topos_frame_input* in;
    uint32_t qp_min, qp_max, window;
    uint8_t known[TC_QP_MAX + 1u];
    int32_t rc[TC_QP_MAX + 1u];       /* per-frame status of the probe */
    uint32_t bytes[TC_QP_MAX + 1u];   /* exact packet size (reference probe count) */
    uint32_t slot[TC_QP_MAX + 1u];
    tcg_enc_result res[TC_QP_MAX + 1u];
    uint32_t slices;
    size_t cap;
} size_table;

/* Encodes qp q and up to window-1 of the nearest unprobed qps of
 * [qp_min, qp_max] in one launch sequence. A call-level failure is returned;
 * per-qp statuses land in the table. */
static int32_t table_fill(size_table* t, uint32_t q)
{
    uint32_t qs[SIZED_WINDOW];
    uint32_t n = 0;
    qs[n++] = q;
    for (uint32_t d = 1; n < t->window && (q + d <= t->qp_max || q >= t->qp_min + d); ++d) {
        if (q + d <= t->qp_max && !t->known[q + d] && n < t->window) { qs[n++] = q + d; }
        if (q >= t->qp_min + d && !t->known[q - d] && n < t->window) { qs[n++] = q - d; }
    }
    tcg_enc_frame jobs[SIZED_WINDOW];
    size_t caps[SIZED_WINDOW];
    tcg_enc_result res[SIZED_WINDOW];
    uint32_t slots[SIZED_WINDOW];
    for (uint32_t i = 0; i < n; ++i) {
        topos_frame_config c = *t->cfg;
        c.qp_base = (uint8_t)qs[i];
        uint32_t nsl = 0;
        uint8_t qpb = 0;
        const int32_t rc = tc_prepare_encode(&c, t->in, &jobs[i], &nsl, &qpb);
        if (rc != TC_OK) { return rc; }
        t->slices = nsl;
        caps[i] = t->cap;
    }
    const int32_t rc = tcg_sized_encode(t->sess, jobs, n, caps, res, slots);
    if (rc != TC_OK) { return rc; }
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t qi = qs[i];
        const tcg_enc_result* r = &res[i];
        /* the reference's probe counts the bytes whatever their total */
        const uint64_t b = 53u + 17u * (uint64_t)(r->color_slices + r->alpha_slices) + r->color_payload +
                           r->alpha_payload;
        t->known[qi] = 1u;
        t->rc[qi] = r->rc;
        t->bytes[qi] = (uint32_t)b;
        t->slot[qi] = slots[i];
        t->res[qi] = *r;
    }
    return TC_OK;
}

/* Probe of qp q: TC_OK with its exact size, or its error. A counting probe
 * (the reference's exact-count probe from its coefficient cache) reports the
 * size of a packet past the 256 MiB packet limit; a whole-frame probe fails
 * there as the encode does. */
static int32_t table_probe(size_table* t, uint32_t q, int counting, uint32_t* bytes)
{
    if (!t->known[q]) {
        const int32_t rc = table_fill(t, q);
        if (rc != TC_OK) { return rc; }
    }
    const int32_t r = t->rc[q];
    if (r != TC_OK && !(counting && r == TC_ERR_LIMIT_EXCEEDED)) {
        return tc_enc_result_status(r, t->res[q].packet_size, 0u);
    }
    *bytes = t->bytes[q];
    return TC_OK;
}

/* The packet of probed qp q to out (the commit of the reference's final or
 * last probe): stats always, the bytes only when they fit. */
static int32_t table_commit(size_table* t, uint32_t q, uint8_t* out, size_t out_cap, topos_frame_stats* stats)
{
    uint32_t b = 0;
    int32_t rc = table_probe(t, q, 0, &b);
    if (rc != TC_OK) { return rc; }
    const tcg_enc_result* r = &t->res[q];
    memset(stats, 0, sizeof(*stats));
    stats->struct_size = (uint32_t)sizeof(topos_frame_stats);
    stats->abi_version = TOPOS_CODEC_ABI_VERSION;
    tc_fill_enc_stats(stats, r, t->slices, (uint8_t)q);
    if ((size_t)r->packet_size > out_cap) {
        return tc_fail(TC_ERR_BUFFER_TOO_SMALL, "out_cap %zu < %zu bytes needed", out_cap, (size_t)r->packet_size);
    }
    if (out != NULL && r->packet_size > 0u) {
        rc = tcg_sized_fetch(t->sess, t->slot[q], out, r->packet_size);
        if (rc == 1) {
            /* the packet was dropped by later probe launches: encode it alone again */
            t->known[q] = 0u;
            const uint32_t w = t->window;
            t->window = 1u;
            rc = table_fill(t, q);
            t->window = w;
            if (rc == TC_OK) { rc = tcg_sized_fetch(t->sess, t->slot[q], out, r->packet_size); }
        }
        if (rc != TC_OK) { return rc < 0 ? rc : tc_fail(TC_ERR_INVALID_ARGUMENT, "sized packet lost"); }
    }
    return TC_OK;
}

/* --------------------------------------------------------------- probe log */

/* reference: codec.c:7271-7289 (sized_probe_ctx) */
typedef struct probe_log {
    size_table* t;
    uint32_t target, qp_min, qp_max;
    uint32_t pts_qp[SIZED_MAX_PTS], pts_bytes[SIZED_MAX_PTS], npts;
    uint32_t budget;
    int violated;
    uint32_t last_qp;
    int has_last;
    int m7;
} probe_log;

/* reference: codec.c:7303-7351 (sized_encode_at): one probe, its point
 * recorded and checked against the earlier ones for monotonicity */
static int32_t encode_at(probe_log* c, uint32_t qp)
{
    if (c->budget == 0u) {
        c->violated = 1;
        return TC_ERR_LIMIT_EXCEEDED;
    }
    uint32_t b = 0;
    const int32_t rc = table_probe(c->t, qp, c->m7, &b);
    count_encode();
    c->budget--;
    c->last_qp = qp;
    c->has_last = 1;
    if (rc < 0) { return rc; }
    for (uint32_t i = 0; i < c->npts; ++i) {
        if (c->pts_qp[i] < qp && c->pts_bytes[i] < b) { c->violated = 1; }
        if (c->pts_qp[i] > qp && c->pts_bytes[i] > b) { c->violated = 1; }
    }
    c->pts_qp[c->npts] = qp;
    c->pts_bytes[c->npts] = b;
    c->npts++;
    return TC_OK;
}

static int bytes_at(const probe_log* c, uint32_t qp, uint32_t* out)
{
    for (uint32_t i = 0; i < c->npts; ++i) {
        if (c->pts_qp[i] == qp) {
            *out = c->pts_bytes[i];
            return 1;
        }
    }
    return 0;
}

/* reference: codec.c:7375-7398 (sized_fit_slope, r6 search) */
static double fit_slope(const probe_log* c)
{
    for (uint32_t i = c->npts; i-- > 1u;) {
        const uint32_t q1 = c->pts_qp[i], b1 = c->pts_bytes[i];
        for (uint32_t j = i; j-- > 0u;) {
            const uint32_t q0 = c->pts_qp[j], b0 = c->pts_bytes[j];
            if (q1 > q0 && b0 > b1 && b0 > 0u) {
                const double dr = log2((double)b0 / (double)b1);
                if (dr > 0.05) {
                    double s = (double)(q1 - q0) / dr;
                    s = s < 1.0 ? 1.0 : (s > 16.0 ? 16.0 : s);
                    return s;
                }
            }
        }
    }
    return 4.0;
}

/* reference: codec.c:7554-7572 (strict_slope_from_pts) */
static double strict_slope(const probe_log* c, double def)
{
    for (uint32_t i = c->npts; i-- > 1u;) {
        const uint32_t q1 = c->pts_qp[i], b1 = c->pts_bytes[i];
        for (uint32_t j = i; j-- > 0u;) {
            const uint32_t q0 = c->pts_qp[j], b0 = c->pts_bytes[j];
            if (q1 > q0 && b0 > b1 && b1 > 0u) {
                const double dr = log2((double)b0 / (double)b1);
                if (dr > 0.05) {
                    double s = (double)(q1 - q0) / dr;
                    s = s < 1.0 ? 1.0 : (s > 16.0 ? 16.0 : s);
                    return s;
                }
            }
        }
    }
    return def;
}

static uint32_t clamp_u32(uint32_t v, uint32_t lo, uint32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ------------------------------------------------------------------ searches */

/* reference: codec.c:7199-7262. Coarse +8 steps then +1 steps up while over
 * the target; then, while under 3/4 of it, one qp down at a time, undoing a
 * step that overshoots. The last probe's packet is the answer. */
static int32_t search_linear(size_table* t, uint32_t qp_base, uint32_t target, uint32_t qp_min, uint32_t qp_max,
                             uint8_t* qp_used, uint8_t* out, size_t out_cap, topos_frame_stats* sp)
{
    uint32_t qp = clamp_u32(qp_base, qp_min, qp_max);
    uint32_t iters = 0u;
    const uint32_t max_iters = 24u;
    uint32_t size = 0u;
    int32_t rc = table_probe(t, qp, 0, &size);
    count_encode();
    iters++;
    while (rc >= 0 && size > target && qp + 8u <= qp_max && iters < max_iters) {
        qp += 8u;
        rc = table_probe(t, qp, 0, &size);
        count_encode();
        iters++;
    }
    while (rc >= 0 && size > target && qp < qp_max && iters < max_iters) {
        qp += 1u;
        rc = table_probe(t, qp, 0, &size);
        count_encode();
        iters++;
    }
    while (rc >= 0 && size <= target && (uint64_t)size * 4u < (uint64_t)target * 3u && qp > qp_min &&
           iters < max_iters) {
        const uint32_t cand = qp - 1u;
        uint32_t s2 = 0u;
        const int32_t rc2 = table_probe(t, cand, 0, &s2);
        count_encode();
        iters++;
        if (rc2 >= 0 && s2 <= target) {
            qp = cand;
            size = s2;
            rc = rc2;
            continue;
        }
        rc = table_probe(t, qp, 0, &size); /* back to the last packet that fitted */
        count_encode();
        iters++;
        break;
    }
    if (rc >= 0) { rc = table_commit(t, qp, out, out_cap, sp); }
    if (qp_used != NULL) { *qp_used = (uint8_t)qp; }
    return rc;
}

/* reference: codec.c:7404-7552. The linear search's upward steps probe for
 * probe; its downward reclaim is found by interpolation and bisection; a
 * search the linear one would have cut off at 24 encodes falls back to it. */
static int32_t search_fast(probe_log* c, uint32_t qp_base, uint8_t* qp_used, uint8_t* out, size_t out_cap,
                           topos_frame_stats* sp, int* fallback)
{
    const uint32_t target = c->target, qp_min = c->qp_min, qp_max = c->qp_max;
    const uint32_t q0 = clamp_u32(qp_base, qp_min, qp_max);
    uint32_t q_final = q0;
    uint32_t size = 0u;
    int32_t rc = encode_at(c, q0);
    if (rc < 0 || c->violated) { goto done; }
    (void)bytes_at(c, q0, &size);
    uint32_t qp = q0, iters = 1u;
    while (rc >= 0 && size > target && qp + 8u <= qp_max && iters < 24u) {
        qp += 8u;
        rc = encode_at(c, qp);
        if (rc < 0 || c->violated) { goto done; }
        (void)bytes_at(c, qp, &size);
        iters++;
    }
    while (rc >= 0 && size > target && qp < qp_max && iters < 24u) {
        qp += 1u;
        rc = encode_at(c, qp);
        if (rc < 0 || c->violated) { goto done; }
        (void)bytes_at(c, qp, &size);
        iters++;
    }
    const uint32_t q_a = qp;
    q_final = q_a;
    int restore_extra = 0;
    {
        uint32_t ba = 0;
        (void)bytes_at(c, q_a, &ba);
        const int fits_a = ba <= target;
        const int p_a = (uint64_t)ba * 4u < (uint64_t)target * 3u;
        if (fits_a && p_a && q_a > qp_min && iters < 24u) {
            uint32_t lo = q_a, hi = 0;
            int have_notp = 0;
            for (;;) {
                uint32_t next;
                if (!have_notp) {
                    double dist = fit_slope(c) * log2((0.75 * (double)target) / (double)ba);
                    if (dist < 0.0) { dist = 0.0; }
                    const uint32_t d = (uint32_t)(dist + 0.999);
                    next = clamp_u32(lo - d - 1u, qp_min, lo - 1u);
                } else {
                    next = (hi + lo) / 2u;
                    if (next == hi) { next = hi + 1u; }
                    if (next >= lo) { next = lo - 1u; }
                }
                rc = encode_at(c, next);
                if (rc < 0 || c->violated) { goto done; }
                uint32_t bn = 0;
                (void)bytes_at(c, next, &bn);
                const int p_n = (uint64_t)bn * 4u < (uint64_t)target * 3u;
                if (p_n) {
                    lo = next;
                    ba = bn;
                    if (lo == qp_min) { break; }
                } else {
                    have_notp = 1;
                    hi = next;
                    if (hi + 1u == lo) { break; }
                }
                if (have_notp && hi + 1u >= lo) { break; }
                if (!have_notp && lo == qp_min) { break; }
            }
            if (have_notp) {
                uint32_t bc = 0;
                (void)bytes_at(c, hi, &bc);
                if (bc <= target) {
                    q_final = hi;
                } else {
                    q_final = hi + 1u;
                    restore_extra = 2;
                }
            } else {
                q_final = qp_min;
            }
        }
    }
    {
        uint32_t iters_check = iters;
        if (q_final < q_a) { iters_check += q_a - q_final; }
        iters_check += (uint32_t)restore_extra;
        if (iters_check > 24u) {
            c->violated = 1;
            goto done;
        }
    }
    if (c->m7 != 0) {
        count_encode(); /* the reference's final encode from its coefficient cache */
    } else if (!c->has_last || c->last_qp != q_final) {
        rc = encode_at(c, q_final);
        if (rc < 0 || c->violated) { goto done; }
    }
    rc = table_commit(c->t, q_final, out, out_cap, sp);
done:
    if (c->violated != 0) {
        *fallback = 1;
        return TC_OK;
    }
    if (qp_used != NULL) { *qp_used = (uint8_t)q_final; }
    return rc;
}

/* reference: codec.c:7578-7787. The smallest qp of [qp_min, qp_max] whose
 * packet fits: slope jumps from a seed (the cross-call hint, else qp_base)
 * until the answer is bracketed, then log interpolation inside the bracket.
 * A probe budget of 24, monotonic sizes and the coefficient cache are its
 * preconditions; without one it falls back to the linear search. */
static int32_t search_strict(probe_log* c, sized_hint* e, uint32_t qp_base, uint8_t* qp_used, uint8_t* out,
                             size_t out_cap, topos_frame_stats* sp, int* fallback)
{
    const uint32_t target = c->target, qp_min = c->qp_min, qp_max = c->qp_max;
    if (c->m7 == 0) {
        *fallback = 1;
        return TC_OK;
    }
    uint32_t q0 = qp_base;
    const int hint_on = atomic_load(&g_hint_disable) == 0;
    const int model_on = atomic_load(&g_hint_model_disable) == 0;
    if (hint_on && e->valid != 0) {
        q0 = e->q;
        if (model_on && e->bytes > 0u && target > 0u) {
            const double dr = log2((double)e->bytes / (double)target);
            double slope = 0.0;
            if (e->prev_bytes > 0u && e->prev != e->q) {
                const uint32_t q_hi = e->q > e->prev ? e->q : e->prev;
                const uint32_t q_lo = q_hi == e->q ? e->prev : e->q;
                const uint32_t b_hi = q_hi == e->q ? e->bytes : e->prev_bytes;
                const uint32_t b_lo = q_hi == e->q ? e->prev_bytes : e->bytes;
                if (q_hi > q_lo && b_lo > b_hi && b_hi > 0u) {
                    slope = (double)(q_hi - q_lo) / log2((double)b_lo / (double)b_hi);
                }
            }
            if (slope > 0.0) {
                slope = slope < 0.25 ? 0.25 : (slope > 32.0 ? 32.0 : slope);
            } else {
                slope = 8.0;
            }
            double dq = slope * dr;
            dq = dq > 32.0 ? 32.0 : (dq < -32.0 ? -32.0 : dq);
            const double q_seed = (double)q0 + dq;
            q0 = q_seed > 0.0 ? (uint32_t)(q_seed + 0.5) : 0u;
        }
    }
    q0 = clamp_u32(q0, qp_min, qp_max);
    int have_lo = 0, have_hi = 0;
    uint32_t lo = 0u, hi = 0u, q_final = qp_max;
    double prior_slope = 4.0;
    if (model_on && e->bytes > 0u && e->prev_bytes > 0u && e->prev != e->q) {
        const uint32_t q_hi = e->q > e->prev ? e->q : e->prev;
        const uint32_t q_lo = q_hi == e->q ? e->prev : e->q;
        const uint32_t b_hi = q_hi == e->q ? e->bytes : e->prev_bytes;
        const uint32_t b_lo = q_hi == e->q ? e->prev_bytes : e->bytes;
        if (q_hi > q_lo && b_lo > b_hi && b_hi > 0u) {
            double s = (double)(q_hi - q_lo) / log2((double)b_lo / (double)b_hi);
            prior_slope = s < 1.0 ? 1.0 : (s > 16.0 ? 16.0 : s);
        }
    }
    int32_t rc = encode_at(c, q0);
    if (rc < 0 || c->violated) { goto done; }
    {
        uint32_t b0 = 0u;
        (void)bytes_at(c, q0, &b0);
        if (b0 <= target) {
            lo = q0;
            have_lo = 1;
        } else {
            hi = q0;
            have_hi = 1;
        }
    }
    for (;;) {
        if (have_lo && (!have_hi ? (lo == qp_min) : (lo == hi + 1u))) {
            q_final = lo;
            break;
        }
        if (have_hi && !have_lo && hi == qp_max) {
            q_final = qp_max; /* nothing fits: the largest qp, best effort */
            break;
        }
        if (c->budget == 0u) {
            c->violated = 1;
            break;
        }
        uint32_t q;
        if (!have_lo) {
            uint32_t bh = 0u;
            (void)bytes_at(c, hi, &bh);
            const double dr = target > 0u && bh > target ? log2((double)bh / (double)target) : 16.0;
            const double slope = strict_slope(c, prior_slope);
            uint32_t dq = (uint32_t)(slope * dr + 0.999);
            dq = dq < 1u ? 1u : (dq > 32u ? 32u : dq);
            q = hi + dq;
            if (q >= qp_max) { q = qp_max; }
        } else if (!have_hi) {
            uint32_t bl = 0u;
            (void)bytes_at(c, lo, &bl);
            const double dr = bl > 0u && (double)target > (double)bl ? log2((double)target / (double)bl) : 16.0;
            const double slope = strict_slope(c, prior_slope);
            uint32_t dq = (uint32_t)(slope * dr + 0.999);
            dq = dq < 1u ? 1u : (dq > 32u ? 32u : dq);
            q = (dq < lo) ? lo - dq : qp_min;
            if (q < qp_min) { q = qp_min; }
            if (q >= lo) { q = lo - 1u; }
        } else {
            uint32_t bh = 0u, bl = 0u;
            (void)bytes_at(c, hi, &bh);
            (void)bytes_at(c, lo, &bl);
            double q_pred;
            if (bh > 0u && bl > 0u && bh > bl) {
                q_pred = (double)hi + ((double)lo - (double)hi) *
                                          (log2((double)bh) - log2((double)(target > 0u ? target : 1u))) /
                                          (log2((double)bh) - log2((double)bl));
            } else {
                q_pred = (double)((hi + lo) / 2u);
            }
            q = (uint32_t)(q_pred + 0.5);
            if (q <= hi) { q = hi + 1u; }
            if (q >= lo) { q = lo - 1u; }
            uint32_t dummy = 0u;
            if (bytes_at(c, q, &dummy)) {
                uint32_t mid = (hi + lo) / 2u;
                if (mid <= hi || mid >= lo) { mid = hi + 1u; }
                q = mid;
                for (; q < lo; ++q) {
                    if (!bytes_at(c, q, &dummy)) { break; }
                }
                if (q >= lo) {
                    q_final = lo;
                    break;
                }
            }
        }
        rc = encode_at(c, q);
        if (rc < 0 || c->violated) { break; }
        uint32_t b = 0u;
        (void)bytes_at(c, q, &b);
        if (b <= target) {
            if (!have_lo || q < lo) { lo = q; }
            have_lo = 1;
        } else {
            if (!have_hi || q > hi) { hi = q; }
            have_hi = 1;
        }
    }
done:
    if (c->violated != 0) {
        *fallback = 1;
        return TC_OK;
    }
    if (rc < 0) { return rc; }
    rc = table_commit(c->t, q_final, out, out_cap, sp);
    count_encode();
    if (rc < 0) { return rc; }
    if (qp_used != NULL) { *qp_used = (uint8_t)q_final; }
    {
        uint32_t bf = 0u;
        if (bytes_at(c, q_final, &bf) != 0) {
            if (e->valid != 0 && e->q != q_final) {
                e->prev = e->q;
                e->prev_bytes = e->bytes;
            }
            e->q = q_final;
            e->valid = 1;
            e->bytes = bf;
        }
    }
    return rc;
}

/* ----------------------------------------------------------------- entry */

/* One size-targeted encode. process_hint: use the process-wide hint record
 * when it is free (the single call), else an empty one (batch workers). */
static int32_t sized_one(const topos_frame_config* cfg, const topos_frame_input* input, uint32_t target_bytes,
                         uint8_t qp_min, uint8_t qp_max, uint8_t* qp_used, uint8_t* out, size_t out_cap,
                         topos_frame_stats* stats, int process_hint)
{
    int32_t rc = tc_frame_config_validate(cfg);
    if (rc != TC_OK) { return rc; }
    if ((cfg->reserved[0] & 0xFFu) == 9u) {
        return tc_fail(TC_ERR_NOT_IMPLEMENTED, "v8 sized encode lands in format-plan batch 2");
    }
    if ((cfg->reserved[0] & 0xFFu) == 10u || (cfg->reserved[0] & 0xFFu) == 11u) {
        return tc_fail(TC_ERR_NOT_IMPLEMENTED,
                       "temporal sized encode is not a write path (fixed anchor-qp P0; use tc_gop_context_encode_frame)");
    }
    if (cfg->pixel_format == 3u) {
        return tc_fail(TC_ERR_NOT_IMPLEMENTED, "TRAW sized rate control is a post-v1 option; use fixed anchor-qp tiers");
    }
    if (qp_min > TC_QP_MAX || qp_max > TC_QP_MAX || qp_min > qp_max) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "qp range %u..%u invalid", (unsigned)qp_min, (unsigned)qp_max);
    }
    topos_frame_stats local;
    memset(&local, 0, sizeof(local));
    topos_frame_stats* sp = stats != NULL ? stats : &local;
    mode_env_init();
    atomic_fetch_add(&g_calls, 1u);

    /* the frame at its own qp: validation of the input exactly as a plain
     * encode, and the geometry that sizes the probe window */
    tcg_enc_frame base;
    uint32_t nsl = 0;
    uint8_t qpb = 0;
    rc = tc_prepare_encode(cfg, input, &base, &nsl, &qpb);
    if (rc != TC_OK) { return rc; }
    uint64_t cblocks = 0, samples = 0;
    for (uint32_t p = 0; p < base.planes; ++p) {
        samples += (uint64_t)base.plane[p].vis_w * base.plane[p].vis_h;
        if (base.plane[p].kind == TCG_PLANE_COLOR) { cblocks += (uint64_t)base.plane[p].cols * base.plane[p].rows; }
    }
    size_table* t = (size_table*)calloc(1, sizeof(size_table));
    if (t == NULL) { return tc_fail(TC_ERR_OUT_OF_MEMORY, "sized encode table"); }
    t->cfg = cfg;
    t->in = input;
    t->qp_min = qp_min;
    t->qp_max = qp_max;
    t->cap = tc_frame_packet_bound(cfg);
    t->window = sized_window(t->cap, samples, cblocks);
    rc = tcg_sized_open(&base, &t->sess);
    if (rc != TC_OK) {
        free(t);
        return rc;
    }

    /* the cross-call hint record: borrowed when free, an empty one otherwise */
    sized_hint fresh;
    memset(&fresh, 0, sizeof(fresh));
    int expected = 0;
    const int borrowed = process_hint && atomic_compare_exchange_strong(&g_hint_busy, &expected, 1);
    sized_hint* e = borrowed ? &g_hint : &fresh;

    probe_log c;
    memset(&c, 0, sizeof(c));
    c.t = t;
    c.target = target_bytes;
    c.qp_min = qp_min;
    c.qp_max = qp_max;
    c.budget = SIZED_PROBE_BUDGET;
    c.m7 = atomic_load(&g_m7_disable) == 0 && cblocks * 256u <= SIZED_FCACHE_MAX_BYTES;

    uint8_t qu = 0;
    int fallback = 0;
    const int mode = atomic_load(&g_mode);
    if (mode == 1) {
        rc = search_linear(t, cfg->qp_base, target_bytes, qp_min, qp_max, &qu, out, out_cap, sp);
    } else {
        rc = mode == 2 ? search_fast(&c, cfg->qp_base, &qu, out, out_cap, sp, &fallback)
                       : search_strict(&c, e, cfg->qp_base, &qu, out, out_cap, sp, &fallback);
        if (fallback != 0) {
            rc = search_linear(t, cfg->qp_base, target_bytes, qp_min, qp_max, &qu, out, out_cap, sp);
        }
    }
    if (borrowed) { atomic_store(&g_hint_busy, 0); }
    tcg_sized_close(t->sess);
    free(t);
    if (qp_used != NULL) { *qp_used = qu; }
    return rc;
}

/* reference: native/src/codec/codec.c:7789-7880 */
TC_EXPORT int32_t tc_frame_encode_sized(const topos_frame_config* cfg, const topos_frame_input* input,
                                        uint32_t target_bytes, uint8_t qp_min, uint8_t qp_max, uint8_t* qp_used,
                                        uint8_t* out, size_t out_cap, topos_frame_stats* stats)
{
    return sized_one(cfg, input, target_bytes, qp_min, qp_max, qp_used, out, out_cap, stats, 1);
}

/* ------------------------------------------------------------------ batch */

typedef struct sized_batch {
    const topos_frame_config* cfgs;
    const topos_frame_input* inputs;
    const uint32_t* targets;
    uint8_t qp_min, qp_max;
    uint8_t* qp_used;
    uint8_t* const* outs;
    const size_t* caps;
    topos_frame_stats* stats;
    int32_t* rcs;
    uint32_t count;
    atomic_uint next;
} sized_batch;

static void* sized_worker(void* arg)
{
    sized_batch* b = (sized_batch*)arg;
    for (;;) {
        const uint32_t i = atomic_fetch_add(&b->next, 1u);
        if (i >= b->count) { break; }
        uint8_t q = 0;
        b->rcs[i] = sized_one(&b->cfgs[i], &b->inputs[i], b->targets[i], b->qp_min, b->qp_max, &q,
                              b->outs[i], b->outs[i] == NULL ? 0u : b->caps[i],
                              b->stats != NULL ? &b->stats[i] : NULL, 0);
        if (b->qp_used != NULL) { b->qp_used[i] = q; }
    }
    return NULL;
}

/* extension: many size-targeted encodes at once. Every frame is searched as a
 * single call made with an empty cross-call hint record (the reference's
 * behaviour when its record is held by another call), so results do not
 * depend on the order of the frames; up to six searches run side by side,
 * each on its own context, and their probe launches overlap on the GPU. */
TC_EXPORT int32_t tcg_frame_encode_sized_batch(const topos_frame_config* cfgs, const topos_frame_input* inputs,
                                               uint32_t count, const uint32_t* target_bytes, uint8_t qp_min,
                                               uint8_t qp_max, uint8_t* qp_used, uint8_t* const* outs,
                                               const size_t* out_caps, topos_frame_stats* stats, int32_t* rcs)
{
    if (count == 0u) { return TC_OK; }
    if (cfgs == NULL || inputs == NULL || target_bytes == NULL || outs == NULL || out_caps == NULL || rcs == NULL) {
        return tc_fail(TC_ERR_INVALID_ARGUMENT, "batch arguments NULL");
    }
    if (count > TC_BATCH_MAX_FRAMES) { return tc_fail(TC_ERR_LIMIT_EXCEEDED, "batch count %u", count); }
    sized_batch b;
    memset(&b, 0, sizeof(b));
    b.cfgs = cfgs;
    b.inputs = inputs;
    b.targets = target_bytes;
    b.qp_min = qp_min;
    b.qp_max = qp_max;
    b.qp_used = qp_used;
    b.outs = outs;
    b.caps = out_caps;
    b.stats = stats;
    b.rcs = rcs;
    b.count = count;
    atomic_init(&b.next, 0u);
    /* searches side by side: bounded by the device bytes of their probe
     * windows, against the smaller of a fixed budget and 3/4 of free memory */
    uint32_t workers = count < SIZED_BATCH_WORKERS ? count : SIZED_BATCH_WORKERS;
    {
        /* the first frame's geometry, counted as four full planes */
        const size_t cap = tc_frame_packet_bound(&cfgs[0]);
        const uint64_t px = (uint64_t)cfgs[0].visible_width * cfgs[0].visible_height;
        const uint64_t samples = px * 4u, cblocks = px / 16u;
        const uint64_t per = (uint64_t)sized_window(cap, samples, cblocks) * ((uint64_t)cap + samples * 2u + cblocks * 2048u);
        uint64_t free_b = 0, total_b = 0;
        tcg_mem_info(&free_b, &total_b);
        if (total_b > 0u && free_b / 4u * 3u < (uint64_t)workers * per) {
            /* idle contexts' buffers from earlier calls are worth more as probe windows */
            tcg_trim_idle();
            tcg_mem_info(&free_b, &total_b);
        }
        uint64_t budget = SIZED_BATCH_BYTES;
        if (total_b > 0u && free_b / 4u * 3u < budget) { budget = free_b / 4u * 3u; }
        const uint64_t fit = per > 0u ? budget / per : workers;
        if (fit < workers) { workers = fit < 1u ? 1u : (uint32_t)fit; }
    }
    pthread_t th[SIZED_BATCH_WORKERS];
    uint32_t started = 0;
    for (uint32_t w = 1; w < workers; ++w) {
        if (pthread_create(&th[started], NULL, sized_worker, &b) == 0) { started++; }
    }
    sized_worker(&b);
    for (uint32_t w = 0; w < started; ++w) { pthread_join(th[w], NULL); }
    /* a search that ran out of device memory beside the others runs again alone */
    for (uint32_t i = 0; i < count; ++i) {
        if (rcs[i] != TC_ERR_OUT_OF_MEMORY) { continue; }
        uint8_t q = 0;
        rcs[i] = sized_one(&cfgs[i], &inputs[i], target_bytes[i], qp_min, qp_max, &q, outs[i],
                           outs[i] == NULL ? 0u : out_caps[i], stats != NULL ? &stats[i] : NULL, 0);
        if (qp_used != NULL) { qp_used[i] = q; }
    }
    for (uint32_t i = 0; i < count; ++i) {
        if (rcs[i] != TC_OK) { return tc_fail(rcs[i], "sized batch: frame %u failed with status %d", i, (int)rcs[i]); }
    }
    return TC_OK;
}
