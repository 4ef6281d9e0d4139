/* CPU oracle: plain-C restatement of the reference JPEG 2000 hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Loaded by tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg as the checker; the product (libgail_b200) never links or calls it.
 *
 * Compiled without fast-math and without floating-point contraction, so every float
 * operation rounds exactly where the reference's x86-64 baseline build rounds.
 * Citations are paths inside the reference project (Josephur/libgail).
 */
#include "gail_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SIGN_BIT 0x80000000u

/* ==================================================================================
 * MQ coder, ISO/IEC 15444-1 Annex C. Probability estimation table C.2 (public standard
 * data; the reference holds the same numbers packed in kernels/mq_table.h:17-65).
 * ================================================================================== */
static const uint16_t k_qe[47] = {0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801,
                                   0x3001, 0x2401, 0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401,
                                   0x3001, 0x2801, 0x2401, 0x2201, 0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101,
                                   0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1, 0x0221, 0x0141, 0x0111, 0x0085,
                                   0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
static const uint8_t k_nmps[47] = {1,  2,  3,  4,  5,  38, 7,  8,  9,  10, 11, 12, 13, 29, 15, 16,
                                   17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32,
                                   33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 45, 46};
static const uint8_t k_nlps[47] = {1,  6,  9,  12, 29, 33, 6,  14, 14, 14, 17, 18, 20, 21, 14, 14,
                                   15, 16, 17, 18, 19, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29,
                                   30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 46};
static const uint8_t k_switch[47] = {1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                     0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

#define CX_RL 17
#define CX_UNI 18
#define NUM_CX 19

/* Initial context states, Table D.7: all 0 except ZC context 0 (4), run-length (3) and
 * uniform (46). mq_init, kernels/mq_encoder.h:48-60. */
static void init_contexts(uint8_t* idx, uint8_t* mps) {
    for (int i = 0; i < NUM_CX; ++i) {
        idx[i] = 0;
        mps[i] = 0;
    }
    idx[0] = 4;
    idx[CX_RL] = 3;
    idx[CX_UNI] = 46;
}

typedef struct {
    uint32_t a, c, b;
    int ct, bp; /* bp: index of the pending byte b; -1 before the first byte out */
    uint8_t* out;
    uint8_t idx[NUM_CX], mps[NUM_CX];
} mq_enc;

typedef struct {
    int bp;
    uint32_t b, c, a;
    int ct;
} mq_snap;

static void mqe_init(mq_enc* e, uint8_t* out) {
    e->a = 0x8000u;
    e->c = 0;
    e->ct = 12;
    e->bp = -1;
    e->b = 0;
    e->out = out;
    init_contexts(e->idx, e->mps);
}

/* BYTEOUT, Figure C.8 (kernels/mq_encoder.h:62-83). */
static void mqe_byteout(mq_enc* e) {
    int stuffed;
    if (e->b == 0xFF) {
        stuffed = 1;
    } else if (e->c < 0x8000000u) {
        stuffed = 0;
    } else {
        e->b += 1; /* carry into the pending byte */
        if (e->b == 0xFF) {
            e->c &= 0x7FFFFFFu;
            stuffed = 1;
        } else {
            stuffed = 0;
        }
    }
    if (e->bp >= 0) e->out[e->bp] = (uint8_t)e->b;
    e->bp += 1;
    if (stuffed) {
        e->b = e->c >> 20;
        e->c &= 0xFFFFFu;
        e->ct = 7;
    } else {
        e->b = (e->c >> 19) & 0xFFu;
        e->c &= 0x7FFFFu;
        e->ct = 8;
    }
}

/* RENORME, Figure C.7. */
static void mqe_renorm(mq_enc* e) {
    do {
        e->a <<= 1;
        e->c <<= 1;
        e->ct -= 1;
        if (e->ct == 0) mqe_byteout(e);
    } while ((e->a & 0x8000u) == 0);
}

/* ENCODE with CODEMPS / CODELPS, Figures C.4-C.6 (kernels/mq_encoder.h:102-118). */
static void mqe_encode(mq_enc* e, int cx, uint32_t d) {
    const int i = e->idx[cx];
    const uint32_t qe = k_qe[i];
    e->a -= qe;
    if (d == e->mps[cx]) {
        if ((e->a & 0x8000u) == 0) {
            if (e->a < qe) e->a = qe;
            else e->c += qe;
            e->idx[cx] = k_nmps[i];
            mqe_renorm(e);
        } else {
            e->c += qe;
        }
    } else {
        if (e->a < qe) e->c += qe;
        else e->a = qe;
        if (k_switch[i]) e->mps[cx] ^= 1u;
        e->idx[cx] = k_nlps[i];
        mqe_renorm(e);
    }
}

static mq_snap mqe_snapshot(const mq_enc* e) {
    mq_snap s;
    s.bp = e->bp;
    s.b = e->b;
    s.c = e->c;
    s.a = e->a;
    s.ct = e->ct;
    return s;
}

/* FLUSH, Figure C.9 with SETBITS (kernels/mq_encoder.h:131-144): returns the length. A
 * final 0xFF byte is not emitted. */
static uint32_t mqe_flush(mq_enc* e) {
    const uint32_t tempc = e->c + e->a;
    e->c |= 0xFFFFu;
    if (e->c >= tempc) e->c -= 0x8000u;
    e->c <<= e->ct;
    mqe_byteout(e);
    e->c <<= e->ct;
    mqe_byteout(e);
    if (e->b != 0xFF) {
        e->out[e->bp] = (uint8_t)e->b;
        return (uint32_t)(e->bp + 1);
    }
    return (uint32_t)e->bp;
}

/* Shortest prefix (>= min_len) of the final codeword after which a decoder that reads
 * 1-bits past the end recovers every decision coded before the snapshot; never ends on
 * 0xFF (mq_trunc_len, kernels/mq_encoder.h:146-169).
 *
 * Fixed point with 16 fraction bits relative to the pending byte at the snapshot: the
 * coded interval is [low, low + A). A prefix whose value is P, with T the weight of its
 * last bit, is decoded as a value approaching P + T from below, which must land in
 * (low, high]. Bytes after an 0xFF carry 7 bits. */
static uint32_t mq_trunc(const mq_snap* s, const uint8_t* buf, uint32_t len, uint32_t min_len) {
    const int base = 43 - s->ct;
    const uint64_t low = ((uint64_t)s->b << base) + ((uint64_t)s->c << 16);
    const uint64_t high = low + ((uint64_t)s->a << 16);
    uint64_t p = 0;
    int used = 0;
    for (int i = s->bp; i < (int)len; ++i) {
        const uint32_t byte = i >= 0 ? buf[i] : 0u;
        const int sh = base - used;
        if (sh < 0) break;
        p += (uint64_t)byte << sh;
        const uint64_t tail = (uint64_t)1 << sh;
        const uint32_t l = (uint32_t)(i + 1);
        if (l >= min_len && byte != 0xFF && p + tail <= high && p + tail > low) return l;
        used += byte == 0xFF ? 7 : 8;
    }
    return len;
}

/* ==================================================================================
 * EBCOT Tier-1 contexts, Annex D.
 * ================================================================================== */
/* Zero coding, Table D.1; orient 0 LL, 1 HL, 2 LH, 3 HH (t1_zc_ctx, kernels/t1_common.h:20-38). */
static int zc_context(int h, int v, int d, int orient) {
    if (orient == 3) {
        const int hv = h + v;
        if (d >= 3) return 8;
        if (d == 2) return hv >= 1 ? 7 : 6;
        if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
        return hv >= 2 ? 2 : hv;
    }
    if (orient == 1) { /* HL: the horizontally high-pass band swaps the roles */
        const int t = h;
        h = v;
        v = t;
    }
    if (h == 2) return 8;
    if (h == 1) {
        if (v >= 1) return 7;
        return d >= 1 ? 6 : 5;
    }
    if (v == 2) return 4;
    if (v == 1) return 3;
    if (d >= 2) return 2;
    return d;
}

/* Sign coding, Table D.3 (t1_sc_ctx, kernels/t1_common.h:41-47): context and the bit the
 * sign is XORed with. hc, vc already clamped to -1..1. */
static void sc_context(int hc, int vc, int* cx, uint32_t* xorbit) {
    static const int ctx[3][3] = {{13, 12, 11}, {10, 9, 10}, {11, 12, 13}}; /* [hc+1 reversed][vc] */
    static const uint8_t xr[3][3] = {{0, 0, 0}, {0, 0, 1}, {1, 1, 1}};
    /* rows: hc = 1, 0, -1; columns: vc = 1, 0, -1 */
    const int r = 1 - hc, c = 1 - vc;
    *cx = ctx[r][c];
    *xorbit = xr[r][c];
}

/* Distortion reductions in units of (2^p delta)^2 / 4096 (t1_dist_sig / t1_dist_ref,
 * kernels/t1_common.h:49-53). w: the 7 magnitude bits from bit p (fraction included). */
static int32_t dist_sig(uint32_t w) { return 192 * (int32_t)w - 9216; }
static int32_t dist_ref(uint32_t w) { return w >= 64u ? 64 * (int32_t)w - 5120 : 3072 - 64 * (int32_t)w; }

enum { FL_SIG = 1, FL_NEG = 2, FL_CODED = 4, FL_REFINED = 8 };

typedef struct {
    const uint32_t* c;
    int w, h, orient, stride;
    uint8_t fl[34 * 34];
    mq_enc mq;
    int32_t dist;
    uint32_t nsym;
    int track;
    float thresh, dscale;
    uint32_t n0[NUM_CX], n1[NUM_CX];
} t1_coder;

static inline uint8_t* cell(t1_coder* t, int x, int y) { return &t->fl[(y + 1) * t->stride + x + 1]; }
static inline int sigat(t1_coder* t, int x, int y) { return *cell(t, x, y) & FL_SIG; }
static inline int chi(t1_coder* t, int x, int y) {
    const uint8_t f = *cell(t, x, y);
    return (f & FL_SIG) ? ((f & FL_NEG) ? -1 : 1) : 0;
}
static inline uint32_t magat(t1_coder* t, int x, int y) { return t->c[y * OR_CBLK + x] & ~SIGN_BIT; }
static inline uint32_t bitat(t1_coder* t, int x, int y, int p) { return (magat(t, x, y) >> (p + OR_FRAC_BITS)) & 1u; }

static void counts(t1_coder* t, int x, int y, int* h, int* v, int* d) {
    *h = sigat(t, x - 1, y) + sigat(t, x + 1, y);
    *v = sigat(t, x, y - 1) + sigat(t, x, y + 1);
    *d = sigat(t, x - 1, y - 1) + sigat(t, x + 1, y - 1) + sigat(t, x - 1, y + 1) + sigat(t, x + 1, y + 1);
}
static int any_neighbour(t1_coder* t, int x, int y) {
    int h, v, d;
    counts(t, x, y, &h, &v, &d);
    return h + v + d;
}

static void code(t1_coder* t, int cx, uint32_t d) {
    mqe_encode(&t->mq, cx, d);
    t->nsym++;
    if (t->track) {
        if (d) t->n1[cx]++;
        else t->n0[cx]++;
    }
}

static int clamp1(int v) { return v < -1 ? -1 : (v > 1 ? 1 : v); }

/* A sample's first 1-bit is in plane p: code its sign, mark it, add its distortion
 * reduction (becomeSig, core/t1_ref.cpp:177-190). */
static void make_significant(t1_coder* t, int x, int y, int p) {
    const int hc = clamp1(chi(t, x - 1, y) + chi(t, x + 1, y));
    const int vc = clamp1(chi(t, x, y - 1) + chi(t, x, y + 1));
    int cx;
    uint32_t xr;
    sc_context(hc, vc, &cx, &xr);
    const uint32_t neg = (*cell(t, x, y) & FL_NEG) ? 1u : 0u;
    code(t, cx, neg ^ xr);
    *cell(t, x, y) |= FL_SIG;
    t->dist += dist_sig((magat(t, x, y) >> p) & 0x7Fu);
}

/* Significance propagation, D.3.1 (spp, core/t1_ref.cpp:200-216). */
static void pass_spp(t1_coder* t, int p) {
    for (int y0 = 0; y0 < t->h; y0 += 4) {
        const int y1 = y0 + 4 < t->h ? y0 + 4 : t->h;
        for (int x = 0; x < t->w; ++x)
            for (int y = y0; y < y1; ++y) {
                if (sigat(t, x, y)) continue;
                int h, v, d;
                counts(t, x, y, &h, &v, &d);
                if (h + v + d == 0) continue;
                const uint32_t b = bitat(t, x, y, p);
                code(t, zc_context(h, v, d, t->orient), b);
                *cell(t, x, y) |= FL_CODED;
                if (b) make_significant(t, x, y, p);
            }
    }
}

/* Magnitude refinement, D.3.3 (mrp, core/t1_ref.cpp:218-234). */
static void pass_mrp(t1_coder* t, int p) {
    for (int y0 = 0; y0 < t->h; y0 += 4) {
        const int y1 = y0 + 4 < t->h ? y0 + 4 : t->h;
        for (int x = 0; x < t->w; ++x)
            for (int y = y0; y < y1; ++y) {
                const uint8_t f = *cell(t, x, y);
                if (!(f & FL_SIG) || (f & FL_CODED)) continue;
                const int cx = (f & FL_REFINED) ? 16 : (any_neighbour(t, x, y) ? 15 : 14);
                code(t, cx, bitat(t, x, y, p));
                *cell(t, x, y) |= FL_REFINED;
                t->dist += dist_ref((magat(t, x, y) >> p) & 0x7Fu);
            }
    }
}

/* Cleanup with run-length mode, D.3.4 (cup, core/t1_ref.cpp:236-270). */
static void pass_cup(t1_coder* t, int p) {
    for (int y0 = 0; y0 < t->h; y0 += 4) {
        const int n = t->h - y0 < 4 ? t->h - y0 : 4;
        for (int x = 0; x < t->w; ++x) {
            int r = 0;
            if (n == 4) {
                int quiet = 1;
                for (int k = 0; k < 4 && quiet; ++k) {
                    const uint8_t f = *cell(t, x, y0 + k);
                    if ((f & (FL_SIG | FL_CODED)) || any_neighbour(t, x, y0 + k)) quiet = 0;
                }
                if (quiet) {
                    int first = -1;
                    for (int k = 0; k < 4; ++k)
                        if (bitat(t, x, y0 + k, p)) {
                            first = k;
                            break;
                        }
                    if (first < 0) {
                        code(t, CX_RL, 0);
                        continue;
                    }
                    code(t, CX_RL, 1);
                    code(t, CX_UNI, (uint32_t)first >> 1);
                    code(t, CX_UNI, (uint32_t)first & 1u);
                    make_significant(t, x, y0 + first, p);
                    r = first + 1;
                }
            }
            for (; r < n; ++r) {
                const int y = y0 + r;
                if (*cell(t, x, y) & (FL_SIG | FL_CODED)) continue;
                int h, v, d;
                counts(t, x, y, &h, &v, &d);
                const uint32_t b = bitat(t, x, y, p);
                code(t, zc_context(h, v, d, t->orient), b);
                if (b) make_significant(t, x, y, p);
            }
        }
    }
}

/* Empirical-entropy byte estimate of the plane's decisions; resets the counts
 * (planeBytesEstimate, core/t1_ref.cpp:115-126). */
static float plane_bytes(t1_coder* t) {
    float bits = 0.f;
    for (int cx = 0; cx < NUM_CX; ++cx) {
        const float n0 = (float)t->n0[cx], n1 = (float)t->n1[cx], n = n0 + n1;
        if (n > 0.f) {
            const float l0 = log2f(fmaxf(n0, 0.5f) / n), l1 = log2f(fmaxf(n1, 0.5f) / n);
            bits += -(n0 * l0 + n1 * l1) + 2.f;
        }
        t->n0[cx] = t->n1[cx] = 0;
    }
    return bits * 0.125f + 1.f;
}

/* Squared error left once planes >= p are known, mid-point reconstruction
 * (residualEnergy, core/t1_ref.cpp:128-141). */
static float residual(t1_coder* t, int p) {
    float e = 0.f;
    const float step = exp2f((float)p);
    for (int y = 0; y < t->h; ++y)
        for (int x = 0; x < t->w; ++x) {
            const uint32_t m = magat(t, x, y);
            const float v = (float)m * (1.f / 64.f);
            const uint32_t q = m >> (p + OR_FRAC_BITS);
            const float rec = q == 0 ? 0.f : ((float)q + 0.5f) * step;
            e += (v - rec) * (v - rec);
        }
    return e;
}

/* Early-termination test after plane p (stopAfterPlane, core/t1_ref.cpp:143-151). */
static int stop_after(t1_coder* t, int p, int32_t plane_dist) {
    const float bytes = plane_bytes(t);
    if (p <= 0) return 0;
    const float dabs = (float)plane_dist * exp2f((float)(2 * p)) * (1.f / 4096.f) * t->dscale;
    if (!(dabs < t->thresh * bytes)) return 0;
    return residual(t, p) * t->dscale < t->thresh * bytes;
}

int or_t1_encode(const uint32_t* coeffs, int w, int h, int orient, int max_passes, float slope_thresh,
                 float dist_scale, uint8_t* buf, size_t buf_cap, or_t1_result* out) {
    t1_coder* t = (t1_coder*)calloc(1, sizeof(t1_coder));
    if (!t) return -2;
    t->c = coeffs;
    t->w = w;
    t->h = h;
    t->orient = orient;
    t->stride = w + 2;
    t->track = slope_thresh > 0.f;
    t->thresh = slope_thresh;
    t->dscale = dist_scale;
    uint32_t maxmag = 0;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const uint32_t v = coeffs[y * OR_CBLK + x];
            if (v & SIGN_BIT) *cell(t, x, y) = FL_NEG;
            const uint32_t m = (v & ~SIGN_BIT) >> OR_FRAC_BITS;
            if (m > maxmag) maxmag = m;
        }
    memset(out, 0, sizeof(*out));
    int nbps = 0;
    while (nbps < 32 && (maxmag >> nbps)) ++nbps;
    out->nbps = nbps;
    if (nbps == 0) {
        free(t);
        return 0;
    }
    if (3 * nbps - 2 > OR_MAX_PASSES || buf_cap < (size_t)OR_CBLK_AREA * 4 * nbps + 64) {
        free(t);
        return -1;
    }
    mqe_init(&t->mq, buf);
    mq_snap snaps[OR_MAX_PASSES];
    int np = 0;
    for (int p = nbps - 1; p >= 0 && np < max_passes; --p) {
        int32_t plane_dist = 0;
        for (int type = (p == nbps - 1 ? 2 : 0); type < 3 && np < max_passes; ++type) {
            t->dist = 0;
            if (type == 0) pass_spp(t, p);
            else if (type == 1) pass_mrp(t, p);
            else pass_cup(t, p);
            snaps[np] = mqe_snapshot(&t->mq);
            out->pass_dist[np] = t->dist;
            plane_dist += t->dist;
            ++np;
        }
        for (int i = 0; i < 34 * 34; ++i) t->fl[i] &= (uint8_t)~FL_CODED;
        if (t->track && stop_after(t, p, plane_dist)) break;
    }
    const uint32_t len = mqe_flush(&t->mq);
    out->num_passes = np;
    out->data_len = len;
    out->num_symbols = t->nsym;
    uint32_t prev = 1;
    for (int k = 0; k < np; ++k) {
        const uint32_t l = k == np - 1 ? len : mq_trunc(&snaps[k], buf, len, prev);
        out->pass_len[k] = l;
        if (l > prev) prev = l;
    }
    free(t);
    return 0;
}

/* quantizeCoeff, core/quant.h:20-25. */
uint32_t or_quantize(float v, float inv_delta, uint32_t max_mag) {
    const float a = v < 0 ? -v : v;
    const float q = a * inv_delta * (float)(1 << OR_FRAC_BITS);
    const uint32_t m = q >= (float)max_mag ? max_mag : (uint32_t)q;
    return m | (v < 0 && m >= (1u << OR_FRAC_BITS) ? SIGN_BIT : 0u);
}

/* ==================================================================================
 * 9/7 irreversible wavelet, Annex F (core/dwt_cpu.cpp). Lifting constants: Table F.4.
 * ================================================================================== */
#define A97 (-1.586134342059924)
#define B97 (-0.052980118572961)
#define G97 0.882911075530934
#define D97 0.443506852043971
#define K97 1.230174104914001

/* One lifting step on samples of one parity of a length-n signal (n >= 2) read with a
 * stride; the ends use the whole-sample symmetric mirror (lift, core/dwt_cpu.cpp:24-33). */
static void lift_f(float* x, int st, int n, int parity, float c) {
    for (int i = parity; i < n; i += 2) {
        const float l = i > 0 ? x[(i - 1) * st] : x[1 * st];
        const float r = i + 1 < n ? x[(i + 1) * st] : x[(n - 2) * st];
        x[i * st] += c * (l + r);
    }
}

/* One level along one line (row: st 1, column: st = stride), de-interleaved output
 * (fdwtRow :54-64 / fdwtColumns :66-93). */
static void fwd_line(float* x, int st, int n, float* tmp) {
    if (n < 2) return;
    lift_f(x, st, n, 1, (float)A97);
    lift_f(x, st, n, 0, (float)B97);
    lift_f(x, st, n, 1, (float)G97);
    lift_f(x, st, n, 0, (float)D97);
    const int sn = (n + 1) / 2;
    for (int i = 0; i < sn; ++i) tmp[i] = x[2 * i * st] * (float)(1.0 / K97);
    for (int i = 0; i < n / 2; ++i) tmp[sn + i] = x[(2 * i + 1) * st] * (float)K97;
    for (int i = 0; i < n; ++i) x[i * st] = tmp[i];
}

static void inv_line(float* x, int st, int n, float* tmp) {
    if (n < 2) return;
    const int sn = (n + 1) / 2;
    for (int i = 0; i < sn; ++i) tmp[2 * i] = x[i * st] * (float)K97;
    for (int i = 0; i < n / 2; ++i) tmp[2 * i + 1] = x[(sn + i) * st] * (float)(1.0 / K97);
    lift_f(tmp, 1, n, 0, (float)-D97);
    lift_f(tmp, 1, n, 1, (float)-G97);
    lift_f(tmp, 1, n, 0, (float)-B97);
    lift_f(tmp, 1, n, 1, (float)-A97);
    for (int i = 0; i < n; ++i) x[i * st] = tmp[i];
}

void or_fdwt97_2d(float* plane, int stride, int width, int height, int levels) {
    const int mx = width > height ? width : height;
    float* tmp = (float*)malloc(sizeof(float) * (size_t)mx);
    int w = width, h = height;
    for (int l = 0; l < levels; ++l) {
        for (int x = 0; x < w; ++x) fwd_line(plane + x, stride, h, tmp); /* columns first (F.4.2) */
        for (int y = 0; y < h; ++y) fwd_line(plane + (size_t)y * stride, 1, w, tmp);
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
    free(tmp);
}

void or_idwt97_2d(float* plane, int stride, int width, int height, int levels, int skip) {
    int ws[40], hs[40];
    ws[0] = width;
    hs[0] = height;
    for (int l = 1; l <= levels; ++l) {
        ws[l] = (ws[l - 1] + 1) / 2;
        hs[l] = (hs[l - 1] + 1) / 2;
    }
    const int mx = width > height ? width : height;
    float* tmp = (float*)malloc(sizeof(float) * (size_t)mx);
    for (int l = levels; l > skip; --l) {
        const int w = ws[l - 1], h = hs[l - 1];
        for (int y = 0; y < h; ++y) inv_line(plane + (size_t)y * stride, 1, w, tmp); /* rows, then columns */
        for (int x = 0; x < w; ++x) inv_line(plane + x, stride, h, tmp);
    }
    free(tmp);
}

static void lift_d(double* x, int n, int parity, double c) {
    for (int i = parity; i < n; i += 2) {
        const double l = i > 0 ? x[i - 1] : x[1];
        const double r = i + 1 < n ? x[i + 1] : x[n - 2];
        x[i] += c * (l + r);
    }
}

void or_idwt97_1d_f64(const double* in, double* out, int n) {
    if (n <= 0) return;
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int sn = (n + 1) / 2;
    for (int i = 0; i < sn; ++i) out[2 * i] = in[i] * K97;
    for (int i = 0; i < n / 2; ++i) out[2 * i + 1] = in[sn + i] * (1.0 / K97);
    lift_d(out, n, 0, -D97);
    lift_d(out, n, 1, -G97);
    lift_d(out, n, 0, -B97);
    lift_d(out, n, 1, -A97);
}

/* ==================================================================================
 * Frame geometry and step sizes (core/layout.cpp).
 * ================================================================================== */
/* Energy of the 1-D synthesis basis of a low or high band at `level` (synth1d,
 * core/layout.cpp:19-35). */
static double synth1d(int level, int high) {
    const int n = 64 << level;
    double* sig = (double*)calloc((size_t)n, sizeof(double));
    double* tmp = (double*)calloc((size_t)n, sizeof(double));
    const int band = n >> level;
    sig[high ? band + band / 2 : band / 2] = 1.0;
    for (int l = level; l >= 1; --l) {
        const int len = n >> (l - 1);
        or_idwt97_1d_f64(sig, tmp, len);
        memcpy(sig, tmp, sizeof(double) * (size_t)len);
    }
    double e = 0;
    for (int i = 0; i < n; ++i) e += sig[i] * sig[i];
    free(sig);
    free(tmp);
    return sqrt(e);
}

double or_synthesis_norm(int level, int orient) {
    const int hx = orient == 1 || orient == 3, hy = orient == 2 || orient == 3;
    return synth1d(level, hx) * synth1d(level, hy);
}

/* Inverse ICT column norms (ictSynthesisNorm, core/layout.cpp:54-60), ICT constants from
 * ISO/IEC 15444-1 G.3. */
static double ict_norm(int comp) {
    static const double cols[3][3] = {{1, 1, 1}, {0, -0.34413, 1.772}, {1.402, -0.71414, 0}};
    double e = 0;
    for (int i = 0; i < 3; ++i) e += cols[comp][i] * cols[comp][i];
    return sqrt(e);
}

void or_geometry_counts(int width, int height, int levels, int* num_bands, int* num_cblks) {
    int ws[40], hs[40];
    ws[0] = width;
    hs[0] = height;
    for (int l = 1; l <= levels; ++l) {
        ws[l] = (ws[l - 1] + 1) / 2;
        hs[l] = (hs[l - 1] + 1) / 2;
    }
    int nb = 0, nc = 0;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r <= levels; ++r)
            for (int o = 0; o < (r == 0 ? 1 : 3); ++o) {
                const int orient = r == 0 ? 0 : o + 1, n = r == 0 ? levels : levels - r + 1;
                const int hx = orient == 1 || orient == 3, hy = orient == 2 || orient == 3;
                const int bw = hx ? ws[n - 1] - ws[n] : ws[n], bh = hy ? hs[n - 1] - hs[n] : hs[n];
                nc += ((bw + 31) / 32) * ((bh + 31) / 32);
                ++nb;
            }
    *num_bands = nb;
    *num_cblks = nc;
}

int or_make_layout(int width, int height, int fourk, double base_step, or_band* bands, or_cblk* cblks) {
    const int levels = fourk ? 6 : 5, guard = fourk ? 2 : 1;
    int ws[40], hs[40];
    ws[0] = width;
    hs[0] = height;
    for (int l = 1; l <= levels; ++l) {
        ws[l] = (ws[l - 1] + 1) / 2;
        hs[l] = (hs[l - 1] + 1) / 2;
    }
    int nb = 0, nc = 0;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r <= levels; ++r)
            for (int o = 0; o < (r == 0 ? 1 : 3); ++o) {
                or_band* b = &bands[nb++];
                memset(b, 0, sizeof(*b));
                b->comp = c;
                b->res = r;
                b->orient = r == 0 ? 0 : o + 1;
                b->level = r == 0 ? levels : levels - r + 1;
                const int n = b->level;
                const int hx = b->orient == 1 || b->orient == 3, hy = b->orient == 2 || b->orient == 3;
                b->px0 = hx ? ws[n] : 0;
                b->py0 = hy ? hs[n] : 0;
                b->w = hx ? ws[n - 1] - ws[n] : ws[n];
                b->h = hy ? hs[n - 1] - hs[n] : hs[n];
                b->ncbx = (b->w + 31) / 32;
                b->ncby = (b->h + 31) / 32;
                b->cblk_base = nc;
                for (int cy = 0; cy < b->ncby; ++cy)
                    for (int cx = 0; cx < b->ncbx; ++cx) {
                        or_cblk* k = &cblks[nc++];
                        k->band = nb - 1;
                        k->x0 = cx * 32;
                        k->y0 = cy * 32;
                        k->w = b->w - k->x0 < 32 ? b->w - k->x0 : 32;
                        k->h = b->h - k->y0 < 32 ? b->h - k->y0 : 32;
                    }
                /* step size chosen for equal image-domain MSE (makeLayout :181-210) */
                const double norm = or_synthesis_norm(b->level, b->orient);
                const int rb = 12 + (b->orient == 0 ? 0 : (b->orient == 3 ? 2 : 1));
                const double x = (base_step / norm) / ldexp(1.0, rb);
                int eps = (int)ceil(-log2(x));
                if (ldexp(x, eps) < 1.0) ++eps;
                if (ldexp(x, eps) >= 2.0) --eps;
                int mu = (int)lround((ldexp(x, eps) - 1.0) * 2048.0);
                if (mu >= 2048) {
                    mu = 0;
                    --eps;
                }
                if (eps < 0 || eps > 31) return -1;
                b->eps = eps;
                b->mu = mu;
                b->delta = (float)(ldexp(1.0, rb - eps) * (1.0 + mu / 2048.0));
                b->mb = guard + eps - 1;
                if (b->mb > 22) return -1;
                const double wc = ict_norm(c);
                b->weight = norm * norm * wc * wc;
            }
    return 0;
}

/* ==================================================================================
 * Colour (core/color.cpp, kernels/color_math.h), managed route without tone map.
 * ================================================================================== */
static void invert3(const double m[9], double r[9]) {
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    r[0] = (m[4] * m[8] - m[5] * m[7]) / det;
    r[1] = (m[2] * m[7] - m[1] * m[8]) / det;
    r[2] = (m[1] * m[5] - m[2] * m[4]) / det;
    r[3] = (m[5] * m[6] - m[3] * m[8]) / det;
    r[4] = (m[0] * m[8] - m[2] * m[6]) / det;
    r[5] = (m[2] * m[3] - m[0] * m[5]) / det;
    r[6] = (m[3] * m[7] - m[4] * m[6]) / det;
    r[7] = (m[1] * m[6] - m[0] * m[7]) / det;
    r[8] = (m[0] * m[4] - m[1] * m[3]) / det;
}

/* Linear RGB -> XYZ from the chromaticities (rgbToXyzMatrix, core/color.cpp:62-82).
 * Primaries: ITU-R BT.709 / BT.2020, SMPTE 432 (P3-D65), SMPTE 431 (DCI-P3). */
static void rgb_to_xyz(int pri, double M[9]) {
    static const double xy[4][4][2] = {
        {{0.640, 0.330}, {0.300, 0.600}, {0.150, 0.060}, {0.3127, 0.3290}},
        {{0.708, 0.292}, {0.170, 0.797}, {0.131, 0.046}, {0.3127, 0.3290}},
        {{0.680, 0.320}, {0.265, 0.690}, {0.150, 0.060}, {0.3127, 0.3290}},
        {{0.680, 0.320}, {0.265, 0.690}, {0.150, 0.060}, {0.314, 0.351}},
    };
    if (pri == OR_PRI_XYZ) {
        for (int i = 0; i < 9; ++i) M[i] = (i % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    const double(*c)[2] = xy[pri];
    double P[9], Pi[9], S[3];
    for (int i = 0; i < 3; ++i) {
        P[0 + i] = c[i][0] / c[i][1];
        P[3 + i] = 1.0;
        P[6 + i] = (1.0 - c[i][0] - c[i][1]) / c[i][1];
    }
    const double W[3] = {c[3][0] / c[3][1], 1.0, (1.0 - c[3][0] - c[3][1]) / c[3][1]};
    invert3(P, Pi);
    for (int i = 0; i < 3; ++i) S[i] = Pi[3 * i] * W[0] + Pi[3 * i + 1] * W[1] + Pi[3 * i + 2] * W[2];
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) M[3 * r + k] = P[3 * r + k] * S[k];
}

void or_color_init(or_color* cc, int transfer, int primaries, double sdr_white) {
    for (int i = 0; i < 65536; ++i) {
        const double e = i / 65535.0;
        double nits = 0;
        switch (transfer) {
        case OR_TF_SRGB: nits = (e <= 0.04045 ? e / 12.92 : pow((e + 0.055) / 1.055, 2.4)) * sdr_white; break;
        case OR_TF_LINEAR: nits = e * sdr_white; break;
        case OR_TF_GAMMA26: nits = pow(e, 2.6) * 52.37; break;
        default: nits = pow(e, 2.4) * sdr_white; break; /* BT.1886, and PQ/HLG shown as a 2.4 signal */
        }
        cc->eotf[i] = (float)nits;
    }
    double M[9];
    rgb_to_xyz(primaries, M);
    for (int i = 0; i < 9; ++i) cc->m[i] = (float)M[i];
}

/* X' = floor(4095 (X / 52.37)^(1/2.6) + 0.5), SMPTE ST 428-1 (cm_encode, color_math.h:109-112). */
static float dci_encode(float v) {
    float n = v / 52.37f;
    n = fminf(fmaxf(n, 0.0f), 1.0f);
    return floorf(4095.0f * powf(n, 1.0f / 2.6f) + 0.5f);
}

static int eotf_index(float v) { return (int)floorf(fminf(fmaxf(v, 0.0f), 1.0f) * 65535.0f + 0.5f); }

void or_color_xyz12(const or_color* cc, uint16_t r16, uint16_t g16, uint16_t b16, int out[3]) {
    const float R = cc->eotf[eotf_index(r16 / 65535.f)];
    const float G = cc->eotf[eotf_index(g16 / 65535.f)];
    const float B = cc->eotf[eotf_index(b16 / 65535.f)];
    const float X = cc->m[0] * R + cc->m[1] * G + cc->m[2] * B;
    const float Y = cc->m[3] * R + cc->m[4] * G + cc->m[5] * B;
    const float Z = cc->m[6] * R + cc->m[7] * G + cc->m[8] * B;
    out[0] = (int)dci_encode(X);
    out[1] = (int)dci_encode(Y);
    out[2] = (int)dci_encode(Z);
}

void or_ict_forward(int x, int y, int z, float out[3]) {
    const float fx = (float)x, fy = (float)y, fz = (float)z;
    out[0] = (float)0.299 * fx + (float)0.587 * fy + (float)0.114 * fz;
    out[1] = (float)(-0.16875) * fx + (float)(-0.33126) * fy + (float)0.5 * fz;
    out[2] = (float)0.5 * fx + (float)(-0.41869) * fy + (float)(-0.08131) * fz;
}

void or_color_frame(const or_color* cc, const uint16_t* rgb, int npix, float* p0, float* p1, float* p2, uint16_t* xyz12) {
    for (int i = 0; i < npix; ++i) {
        int c[3];
        float o[3];
        or_color_xyz12(cc, rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2], c);
        if (xyz12) {
            xyz12[3 * i] = (uint16_t)c[0];
            xyz12[3 * i + 1] = (uint16_t)c[1];
            xyz12[3 * i + 2] = (uint16_t)c[2];
        }
        or_ict_forward(c[0] - 2048, c[1] - 2048, c[2] - 2048, o);
        p0[i] = o[0];
        p1[i] = o[1];
        p2[i] = o[2];
    }
}

/* round-half-up of a value in [0, 65535] (roundTo16, core/color.cpp:134-140) */
static uint16_t round16(float v) {
    const int r = (int)v;
    return (uint16_t)(r + ((v - (float)r) >= 0.5f ? 1 : 0));
}
static float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

static float sample(const void* src, int bits, size_t i) {
    return bits > 8 ? (float)((const uint16_t*)src)[i] : (float)((const uint8_t*)src)[i];
}

void or_planar_to_rgb48(const or_planar* f, const void* src, uint16_t* rgb) {
    const int aw = f->active_w, ah = f->active_h;
    const int cw = (aw + f->sx) >> f->sx, ch = (ah + f->sy) >> f->sy;
    const size_t uoff = (size_t)aw * ah, voff = uoff + (size_t)cw * ch;
    const float maxv = (float)((1 << f->bits) - 1), scale = (float)(1 << (f->bits - 8));
    const double kg = 1.0 - f->kr - f->kb;
    const float crR = (float)(2 * (1 - f->kr)), cbB = (float)(2 * (1 - f->kb));
    const float cbG = (float)(2 * f->kb * (1 - f->kb) / kg), crG = (float)(2 * f->kr * (1 - f->kr) / kg);
    memset(rgb, 0, sizeof(uint16_t) * (size_t)f->width * f->height * 3);
    for (int ay = 0; ay < ah; ++ay) {
        float cyp = !f->sy ? (float)ay : f->chroma == 2 ? ay * 0.5f : (ay - 0.5f) * 0.5f;
        cyp = clampf(cyp, 0.f, (float)(ch - 1));
        const int y0 = (int)cyp, y1 = y0 + 1 < ch ? y0 + 1 : ch - 1;
        const float fy = cyp - y0;
        uint16_t* o = rgb + ((size_t)(ay + f->oy) * f->width + f->ox) * 3;
        for (int x = 0; x < aw; ++x, o += 3) {
            float cxp = !f->sx ? (float)x : f->chroma == 1 ? (x - 0.5f) * 0.5f : x * 0.5f;
            cxp = clampf(cxp, 0.f, (float)(cw - 1));
            const int x0 = (int)cxp, x1 = x0 + 1 < cw ? x0 + 1 : cw - 1;
            const float fx = cxp - x0;
            float uv[2];
            for (int k = 0; k < 2; ++k) {
                const size_t off = k ? voff : uoff;
                const float a = sample(src, f->bits, off + (size_t)y0 * cw + x0), b = sample(src, f->bits, off + (size_t)y0 * cw + x1);
                const float c = sample(src, f->bits, off + (size_t)y1 * cw + x0), d = sample(src, f->bits, off + (size_t)y1 * cw + x1);
                uv[k] = (a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy;
            }
            float Y = sample(src, f->bits, (size_t)ay * aw + x), U = uv[0], V = uv[1];
            float v[3];
            if (f->rgb) {
                v[0] = V / maxv;
                v[1] = Y / maxv;
                v[2] = U / maxv;
            } else {
                if (f->full_range) {
                    Y /= maxv;
                    U = (U - 128.f * scale) / maxv;
                    V = (V - 128.f * scale) / maxv;
                } else {
                    Y = (Y - 16.f * scale) / (219.f * scale);
                    U = (U - 128.f * scale) / (224.f * scale);
                    V = (V - 128.f * scale) / (224.f * scale);
                }
                v[0] = Y + crR * V;
                v[1] = Y - cbG * U - crG * V;
                v[2] = Y + cbB * U;
            }
            for (int c = 0; c < 3; ++c) o[c] = round16(clampf(v[c], 0.f, 1.f) * 65535.f);
        }
    }
}

uint16_t or_xyz12_to_16(uint32_t v) {
    if (v > 4095u) v = 4095u;
    return (uint16_t)((v * 65535u + 2047u) / 4095u);
}

/* ==================================================================================
 * Decoder: MQ decoding (C.3) and Tier-1 decoding (core/t1_dec.cpp).
 * ================================================================================== */
typedef struct {
    uint32_t a, c;
    int ct;
    uint32_t bp, end;
    const uint8_t* in;
    uint8_t idx[NUM_CX], mps[NUM_CX];
} mq_dec;

/* Bytes past the end read as 0xFF (C.3.4; mq_decoder.h:40-42). */
static uint32_t dec_at(const mq_dec* d, uint32_t i) { return i < d->end ? d->in[i] : 0xFFu; }

/* BYTEIN, Figure C.19 (mqd_bytein, kernels/mq_decoder.h:46-61). */
static void mqd_bytein(mq_dec* d) {
    const uint32_t b = dec_at(d, d->bp), b1 = dec_at(d, d->bp + 1);
    if (b == 0xFF) {
        if (b1 > 0x8F) {
            d->c += 0xFF00u;
            d->ct = 8;
        } else {
            d->bp += 1;
            d->c += b1 << 9;
            d->ct = 7;
        }
    } else {
        d->bp += 1;
        d->c += b1 << 8;
        d->ct = 8;
    }
}

static void mqd_init(mq_dec* d, const uint8_t* in, uint32_t len) {
    d->in = in;
    d->bp = 0;
    d->end = len;
    d->c = dec_at(d, 0) << 16;
    mqd_bytein(d);
    d->c <<= 7;
    d->ct -= 7;
    d->a = 0x8000u;
    init_contexts(d->idx, d->mps);
}

static void mqd_renorm(mq_dec* d) {
    do {
        if (d->ct == 0) mqd_bytein(d);
        d->a <<= 1;
        d->c <<= 1;
        d->ct -= 1;
    } while ((d->a & 0x8000u) == 0);
}

/* DECODE with MPS/LPS exchange, Figures C.15-C.17. */
static uint32_t mqd_decode(mq_dec* d, int cx) {
    const int i = d->idx[cx];
    const uint32_t qe = k_qe[i];
    uint32_t bit;
    d->a -= qe;
    if ((d->c >> 16) < qe) {
        if (d->a < qe) {
            bit = d->mps[cx];
            d->idx[cx] = k_nmps[i];
        } else {
            bit = d->mps[cx] ^ 1u;
            if (k_switch[i]) d->mps[cx] ^= 1u;
            d->idx[cx] = k_nlps[i];
        }
        d->a = qe;
        mqd_renorm(d);
    } else {
        d->c -= qe << 16;
        if ((d->a & 0x8000u) == 0) {
            if (d->a < qe) {
                bit = d->mps[cx] ^ 1u;
                if (k_switch[i]) d->mps[cx] ^= 1u;
                d->idx[cx] = k_nlps[i];
            } else {
                bit = d->mps[cx];
                d->idx[cx] = k_nmps[i];
            }
            mqd_renorm(d);
        } else {
            bit = d->mps[cx];
        }
    }
    return bit;
}

typedef struct {
    int w, h, orient, stride;
    uint8_t fl[34 * 34];
    mq_dec mq;
    uint32_t* out;
} t1_decoder;

static inline uint8_t* dcell(t1_decoder* t, int x, int y) { return &t->fl[(y + 1) * t->stride + x + 1]; }
static inline int dsig(t1_decoder* t, int x, int y) { return *dcell(t, x, y) & FL_SIG; }
static inline int dchi(t1_decoder* t, int x, int y) {
    const uint8_t f = *dcell(t, x, y);
    return (f & FL_SIG) ? ((f & FL_NEG) ? -1 : 1) : 0;
}
static void dcounts(t1_decoder* t, int x, int y, int* h, int* v, int* d) {
    *h = dsig(t, x - 1, y) + dsig(t, x + 1, y);
    *v = dsig(t, x, y - 1) + dsig(t, x, y + 1);
    *d = dsig(t, x - 1, y - 1) + dsig(t, x + 1, y - 1) + dsig(t, x - 1, y + 1) + dsig(t, x + 1, y + 1);
}

static void dmake_significant(t1_decoder* t, int x, int y, int p) {
    const int hc = clamp1(dchi(t, x - 1, y) + dchi(t, x + 1, y));
    const int vc = clamp1(dchi(t, x, y - 1) + dchi(t, x, y + 1));
    int cx;
    uint32_t xr;
    sc_context(hc, vc, &cx, &xr);
    const uint32_t s = mqd_decode(&t->mq, cx) ^ xr;
    *dcell(t, x, y) |= (uint8_t)(FL_SIG | (s ? FL_NEG : 0));
    t->out[y * OR_CBLK + x] = (s << 31) | (3u << p); /* the bit plus the mid-point below it */
}

static void dpass_spp(t1_decoder* t, int p) {
    for (int y0 = 0; y0 < t->h; y0 += 4) {
        const int y1 = y0 + 4 < t->h ? y0 + 4 : t->h;
        for (int x = 0; x < t->w; ++x)
            for (int y = y0; y < y1; ++y) {
                if (dsig(t, x, y)) continue;
                int h, v, d;
                dcounts(t, x, y, &h, &v, &d);
                if (h + v + d == 0) continue;
                const uint32_t b = mqd_decode(&t->mq, zc_context(h, v, d, t->orient));
                *dcell(t, x, y) |= FL_CODED;
                if (b) dmake_significant(t, x, y, p);
            }
    }
}

static void dpass_mrp(t1_decoder* t, int p) {
    for (int y0 = 0; y0 < t->h; y0 += 4) {
        const int y1 = y0 + 4 < t->h ? y0 + 4 : t->h;
        for (int x = 0; x < t->w; ++x)
            for (int y = y0; y < y1; ++y) {
                const uint8_t f = *dcell(t, x, y);
                if (!(f & FL_SIG) || (f & FL_CODED)) continue;
                int h, v, d;
                dcounts(t, x, y, &h, &v, &d);
                const int cx = (f & FL_REFINED) ? 16 : (h + v + d ? 15 : 14);
                const uint32_t b = mqd_decode(&t->mq, cx);
                *dcell(t, x, y) |= FL_REFINED;
                /* the refinement bit replaces the mid-point guess of the plane above */
                t->out[y * OR_CBLK + x] += b ? (1u << p) : (0u - (1u << p));
            }
    }
}

static void dpass_cup(t1_decoder* t, int p) {
    for (int y0 = 0; y0 < t->h; y0 += 4) {
        const int n = t->h - y0 < 4 ? t->h - y0 : 4;
        for (int x = 0; x < t->w; ++x) {
            int r = 0;
            if (n == 4) {
                int quiet = 1;
                for (int k = 0; k < 4 && quiet; ++k) {
                    int h, v, d;
                    dcounts(t, x, y0 + k, &h, &v, &d);
                    if ((*dcell(t, x, y0 + k) & (FL_SIG | FL_CODED)) || h + v + d) quiet = 0;
                }
                if (quiet) {
                    if (!mqd_decode(&t->mq, CX_RL)) continue;
                    int first = (int)mqd_decode(&t->mq, CX_UNI) << 1;
                    first |= (int)mqd_decode(&t->mq, CX_UNI);
                    dmake_significant(t, x, y0 + first, p);
                    r = first + 1;
                }
            }
            for (; r < n; ++r) {
                const int y = y0 + r;
                if (*dcell(t, x, y) & (FL_SIG | FL_CODED)) continue;
                int h, v, d;
                dcounts(t, x, y, &h, &v, &d);
                if (mqd_decode(&t->mq, zc_context(h, v, d, t->orient))) dmake_significant(t, x, y, p);
            }
        }
    }
}

void or_t1_decode(const uint8_t* data, uint32_t len, int w, int h, int orient, int nbps, int passes, uint32_t* out) {
    t1_decoder* t = (t1_decoder*)calloc(1, sizeof(t1_decoder));
    t->w = w;
    t->h = h;
    t->orient = orient;
    t->stride = w + 2;
    t->out = out;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) out[y * OR_CBLK + x] = 0;
    mqd_init(&t->mq, data, len);
    int done = 0;
    for (int p = nbps - 1; p >= 0 && done < passes; --p) {
        for (int type = (p == nbps - 1 ? 2 : 0); type < 3 && done < passes; ++type, ++done) {
            if (type == 0) dpass_spp(t, p);
            else if (type == 1) dpass_mrp(t, p);
            else dpass_cup(t, p);
        }
        for (int i = 0; i < 34 * 34; ++i) t->fl[i] &= (uint8_t)~FL_CODED;
    }
    free(t);
}

void or_ict_inverse_pack(float y0, float y1, float y2, int shift, uint16_t out[3]) {
    const float v[3] = {y0 + (float)1.402 * y2, y0 + (float)(-0.34413) * y1 + (float)(-0.71414) * y2,
                        y0 + (float)1.772 * y1};
    for (int k = 0; k < 3; ++k) {
        int code = (int)floorf(v[k] + 2048.5f);
        code = code < 0 ? 0 : (code > 4095 ? 4095 : code);
        out[k] = (uint16_t)(code << shift);
    }
}

/* ==================================================================================
 * Batch helpers for the tests (loops over the functions above).
 * ================================================================================== */
int or_t1_encode_many(const uint32_t* coeffs, const int32_t* geom4, uint32_t n, float slope, const float* dscale,
                      uint32_t* info4, uint32_t* pass_len, int32_t* pass_dist, uint8_t* data, uint32_t stride) {
    static uint8_t buf[OR_CBLK_AREA * 4 * 24 + 64];
    for (uint32_t i = 0; i < n; ++i) {
        or_t1_result r;
        const int32_t* g = geom4 + 4 * i;
        if (or_t1_encode(coeffs + (size_t)i * OR_CBLK_AREA, g[0], g[1], g[2], g[3], slope, dscale ? dscale[i] : 1.f, buf,
                         sizeof buf, &r) != 0)
            return -1;
        if (r.data_len > stride) return -2;
        info4[4 * i] = (uint32_t)r.nbps;
        info4[4 * i + 1] = (uint32_t)r.num_passes;
        info4[4 * i + 2] = r.num_symbols;
        info4[4 * i + 3] = r.data_len;
        memcpy(pass_len + (size_t)i * 64, r.pass_len, sizeof r.pass_len);
        memcpy(pass_dist + (size_t)i * 64, r.pass_dist, sizeof r.pass_dist);
        memcpy(data + (size_t)i * stride, buf, r.data_len);
    }
    return 0;
}

/* Dead-zone quantisation of Mallat planes into code-block-major words
 * (quantizeCodeBlock, core/quant.cpp:8-20). */
void or_quantize_frame(const float* planes, int width, int height, const or_band* bands, const or_cblk* cblks, int nc,
                       uint32_t* out) {
    const size_t npix = (size_t)width * height;
    for (int i = 0; i < nc; ++i) {
        const or_cblk* k = &cblks[i];
        const or_band* b = &bands[k->band];
        const float* plane = planes + (size_t)b->comp * npix;
        const float inv = 1.0f / b->delta;
        const uint32_t max_mag = ((1u << b->mb) << OR_FRAC_BITS) - 1u;
        uint32_t* o = out + (size_t)i * OR_CBLK_AREA;
        memset(o, 0, OR_CBLK_AREA * 4);
        for (int y = 0; y < k->h; ++y)
            for (int x = 0; x < k->w; ++x)
                o[y * OR_CBLK + x] = or_quantize(plane[(size_t)(b->py0 + k->y0 + y) * width + b->px0 + k->x0 + x], inv, max_mag);
    }
}

/* The 12-bit code of X / 52.37 = n (cm_encode's arithmetic, color_math.h:109-112). */
int or_dci_code(float n) { return (int)floorf(4095.0f * powf(n, 1.0f / 2.6f) + 0.5f); }
