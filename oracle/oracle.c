/*
 * CPU ORACLE — test infrastructure only.
 *
 * This file restates, in plain C, the reference ExCLucene GPU path's codec and
 * list-format arithmetic and computes exact conjunctive (AND) intersections.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it, and only as the checker: no product code path links or calls it.
 *
 * Pinning: the ParaPFD block codec below is checked byte-for-byte against the
 * reference's own src/gpu/Compressed/include/ParaPFor.cpp compiled from source
 * (oracle/Makefile target `ref`), and the regression fits against the reference
 * getRegressionInfo() functions compiled from source; golden vectors made from
 * those builds are committed under tests/golden/.
 *
 * Build: `make -C oracle` (gcc, -O2 -ffp-contract=off, no -march flags, so the
 * float/double arithmetic matches the reference host code, which nvcc compiled
 * through the default x86-64 host compiler without FMA).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>

#define OR_OK 0
#define OR_E_FORMAT 4
#define OR_E_INVALID 1

/* util.h:24-26 (gccbits) */
static inline uint32_t or_bits(uint32_t v) { return v == 0 ? 0u : 32u - (uint32_t)__builtin_clz(v); }
/* util.h:20-22 */
static inline uint64_t or_roundup32(uint64_t v) { return (v + 31u) / 32u; }

/* pack.h:14-24 — LSB-first bit packing of `bit`-bit values; values are < 2^bit. */
static void or_pack(const uint32_t *in, uint32_t *out, uint32_t bit, uint32_t n) {
    uint64_t nwords = or_roundup32((uint64_t)n * bit);
    memset(out, 0, nwords * sizeof(uint32_t));
    if (bit == 0) return;
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t pos = (uint64_t)i * bit;
        uint64_t idx = pos >> 5;
        uint32_t sh = (uint32_t)(pos & 31u);
        uint64_t v = (uint64_t)in[i] << sh;
        out[idx] |= (uint32_t)v;
        if (sh + bit > 32u) out[idx + 1] |= (uint32_t)(v >> 32);
    }
}

/* unpack.h:14-23 — inverse of or_pack; never reads past the packed words. */
static void or_unpack(const uint32_t *in, uint32_t *out, uint32_t bit, uint32_t n) {
    if (bit == 0) { memset(out, 0, (size_t)n * sizeof(uint32_t)); return; }
    uint64_t mask = (bit == 32) ? 0xffffffffull : ((1ull << bit) - 1ull);
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t pos = (uint64_t)i * bit;
        uint64_t idx = pos >> 5;
        uint32_t sh = (uint32_t)(pos & 31u);
        uint64_t w = in[idx];
        if (sh + bit > 32u) w |= (uint64_t)in[idx + 1] << 32;
        out[i] = (uint32_t)((w >> sh) & mask);
    }
}

/* ParaPFor.cpp:31-53 (tryB / findBestB): smallest b in [0,32) whose exception
 * count satisfies (float)nEx <= FRAC * n, evaluated in single precision. */
static uint32_t or_find_best_b(const uint32_t *in, uint32_t n, float frac) {
    for (uint32_t b = 0; b < 32; ++b) {
        uint32_t nex = 0;
        for (uint32_t i = 0; i < n; ++i)
            if (in[i] >= (1u << b)) ++nex;
        if ((float)nex <= frac * (float)n) return b;
    }
    return 32;
}

/* ParaPFor.cpp:56-94 (encodeBlock). Returns words written, or 0 with *err set
 * when the block is not representable by the descriptor (lb or hb = 32, or
 * more than 65535 exceptions). */
uint32_t or_parapfd_encode_block(const uint32_t *in, uint32_t n, float frac, uint32_t *out, int *err) {
    *err = OR_OK;
    uint32_t lb = or_find_best_b(in, n, frac);
    if (lb >= 32) { *err = OR_E_FORMAT; return 0; }
    uint32_t *lower = (uint32_t *)malloc((size_t)(n ? n : 1) * 4);
    uint32_t *high = (uint32_t *)malloc((size_t)(n ? n : 1) * 4);
    uint32_t *pos = (uint32_t *)malloc((size_t)(n ? n : 1) * 4);
    uint32_t en = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (in[i] >= (1u << lb)) {
            lower[i] = in[i] & ((1u << lb) - 1u);
            high[en] = in[i] >> lb;
            pos[en] = i;
            ++en;
        } else {
            lower[i] = in[i];
        }
    }
    uint32_t w = 1;
    or_pack(lower, out + w, lb, n);
    w += (uint32_t)or_roundup32((uint64_t)n * lb);
    if (en > 0) {
        if (en > 65535u) { *err = OR_E_FORMAT; free(lower); free(high); free(pos); return 0; }
        uint32_t eb = or_bits(pos[en - 1]);
        uint32_t acc = 0;
        for (uint32_t i = 0; i < en; ++i) acc |= high[i];
        uint32_t hb = or_bits(acc);
        if (hb >= 32 || eb >= 32) { *err = OR_E_FORMAT; free(lower); free(high); free(pos); return 0; }
        or_pack(pos, out + w, eb, en);
        w += (uint32_t)or_roundup32((uint64_t)en * eb);
        or_pack(high, out + w, hb, en);
        w += (uint32_t)or_roundup32((uint64_t)en * hb);
        out[0] = (lb << 26) + (eb << 21) + (hb << 16) + en;
    } else {
        out[0] = lb << 26;
    }
    free(lower); free(high); free(pos);
    return w;
}

/* ParaPFor.cpp:101-126 (decodeBlock). Returns words consumed. */
uint32_t or_parapfd_decode_block(const uint32_t *in, uint32_t n, uint32_t *out) {
    uint32_t d = in[0];
    uint32_t lb = (d >> 26) % 32u, eb = (d >> 21) & 31u, hb = (d >> 16) & 31u, en = d & 65535u;
    uint32_t w = 1;
    or_unpack(in + w, out, lb, n);
    w += (uint32_t)or_roundup32((uint64_t)n * lb);
    if (en > 0) {
        uint32_t *pos = (uint32_t *)malloc((size_t)en * 4);
        uint32_t *high = (uint32_t *)malloc((size_t)en * 4);
        or_unpack(in + w, pos, eb, en);
        w += (uint32_t)or_roundup32((uint64_t)en * eb);
        or_unpack(in + w, high, hb, en);
        w += (uint32_t)or_roundup32((uint64_t)en * hb);
        for (uint32_t i = 0; i < en; ++i) out[pos[i]] |= high[i] << lb;
        free(pos); free(high);
    }
    return w;
}

/* ---------------------------------------------------------------------------
 * NewPFD (NewPFor.cpp:52-139) with Simple-16 exception streams (Simple16.h).
 * ------------------------------------------------------------------------- */

/* The 16 Simple-16 layouts, each as up to three (count, width) runs; the
 * values of one word are laid out from bit 0 up, the selector in bits 28-31. */
static const unsigned char OR_S16[16][6] = {
    {28, 1, 0, 0, 0, 0}, {7, 2, 14, 1, 0, 0}, {7, 1, 7, 2, 7, 1}, {14, 1, 7, 2, 0, 0},
    {14, 2, 0, 0, 0, 0}, {1, 4, 8, 3, 0, 0},  {1, 3, 4, 4, 3, 3}, {7, 4, 0, 0, 0, 0},
    {4, 5, 2, 4, 0, 0},  {2, 4, 4, 5, 0, 0},  {3, 6, 2, 5, 0, 0}, {2, 5, 3, 6, 0, 0},
    {4, 7, 0, 0, 0, 0},  {1, 10, 2, 9, 0, 0}, {2, 14, 0, 0, 0, 0}, {1, 28, 0, 0, 0, 0}};

static uint32_t or_s16_width(uint32_t k, uint32_t j) {
    for (int r = 0; r < 3; ++r) {
        if (j < OR_S16[k][2 * r]) return OR_S16[k][2 * r + 1];
        j -= OR_S16[k][2 * r];
    }
    return 0;
}

static uint32_t or_s16_count(uint32_t k) { return (uint32_t)OR_S16[k][0] + OR_S16[k][2] + OR_S16[k][4]; }

/* Simple16.h s16_encode: the first layout that holds the next values.
 * Returns words written or -1 if a value exceeds 28 bits. */
static int64_t or_s16_encode(const uint32_t *v, uint32_t n, uint32_t *out) {
    uint64_t nw = 0;
    uint32_t i = 0;
    while (i < n) {
        uint32_t k;
        for (k = 0; k < 16; ++k) {
            uint32_t c = or_s16_count(k), vol = c < n - i ? c : n - i, j;
            for (j = 0; j < vol; ++j)
                if ((uint64_t)v[i + j] >= (1ull << or_s16_width(k, j))) break;
            if (j == vol) {
                uint32_t word = k << 28, sh = 0;
                for (j = 0; j < vol; ++j) { word |= v[i + j] << sh; sh += or_s16_width(k, j); }
                out[nw++] = word;
                i += vol;
                break;
            }
        }
        if (k == 16) return -1;
    }
    return (int64_t)nw;
}

/* S16_DECODE: n values from the stream; returns words read. */
static uint32_t or_s16_decode(const uint32_t *in, uint32_t n, uint32_t *out) {
    uint32_t r = 0, i = 0;
    while (i < n) {
        uint32_t word = in[r++], k = word >> 28, sh = 0;
        for (uint32_t j = 0; j < or_s16_count(k) && i < n; ++j) {
            uint32_t wd = or_s16_width(k, j);
            out[i++] = (word >> sh) & (wd == 32 ? 0xffffffffu : ((1u << wd) - 1u));
            sh += wd;
        }
    }
    return r;
}

/* NewPFor.cpp:52-108 (encodeBlock). */
uint32_t or_newpfd_encode_block(const uint32_t *in, uint32_t n, float frac, uint32_t *out, int *err) {
    *err = OR_OK;
    uint32_t b = or_find_best_b(in, n, frac);
    if (b >= 32) { *err = OR_E_FORMAT; return 0; }
    uint32_t *lower = (uint32_t *)malloc((size_t)(n ? n : 1) * 4);
    uint32_t *all = (uint32_t *)malloc((size_t)(2 * n + 2) * 4);
    uint32_t *pos = (uint32_t *)malloc((size_t)(n ? n : 1) * 4);
    uint32_t en = 0;
    for (uint32_t i = 0; i < n; ++i) {
        lower[i] = in[i] & ((1u << b) - 1u);
        if (in[i] >= (1u << b)) { pos[en] = i; all[n + en] = in[i] >> b; ++en; }
    }
    uint32_t w = 1;
    or_pack(lower, out + w, b, n);
    w += (uint32_t)or_roundup32((uint64_t)n * b);
    if (en > 65535u) { *err = OR_E_FORMAT; free(lower); free(all); free(pos); return 0; }
    out[0] = (b << 26) + en;
    if (en) {
        /* [first position, later positions as gaps minus one, high parts] */
        uint32_t *seq = (uint32_t *)malloc((size_t)2 * en * 4);
        for (uint32_t i = 0; i < en; ++i) {
            seq[i] = i ? pos[i] - pos[i - 1] - 1u : pos[0];
            seq[en + i] = all[n + i];
        }
        int64_t nw = or_s16_encode(seq, 2 * en, out + w);
        free(seq);
        if (nw < 0) { *err = OR_E_FORMAT; free(lower); free(all); free(pos); return 0; }
        w += (uint32_t)nw;
    }
    free(lower); free(all); free(pos);
    return w;
}

/* NewPFor.cpp:111-132 (decodeBlock). Returns words consumed. */
uint32_t or_newpfd_decode_block(const uint32_t *in, uint32_t n, uint32_t *out) {
    uint32_t b = (in[0] >> 26) % 32u, en = in[0] & 65535u;
    uint32_t w = 1;
    or_unpack(in + w, out, b, n);
    w += (uint32_t)or_roundup32((uint64_t)n * b);
    if (en) {
        uint32_t *seq = (uint32_t *)malloc((size_t)2 * en * 4);
        w += or_s16_decode(in + w, 2 * en, seq);
        uint32_t p = 0;
        for (uint32_t i = 0; i < en; ++i) {
            p = i ? p + seq[i] + 1u : seq[0];
            if (p < n) out[p] += seq[en + i] << b;
        }
        free(seq);
    }
    return w;
}

/* ---------------------------------------------------------------------------
 * Regression fits.
 * ------------------------------------------------------------------------- */

/* SegLRC_Generator.cu:264-331 (also LRCSeg_Generator.cu:261-330 and
 * HS_SegLRC_Generator.cu:292-359, identical bodies): double least squares over
 * (i, y[i]); float slope and intercept; float inverse-distance safe range. */
void or_fit_seg(const uint32_t *y, uint32_t n, float *a, float *b, uint32_t *L, uint32_t *R) {
    if (n == 0) { *a = 1.0f; *b = 0.0f; *L = 0; *R = 0; return; }
    if (n == 1) { *a = 1.0f; *b = (float)y[0]; *L = 0; *R = 0; return; }
    double xa = 0, ya = 0;
    for (uint32_t i = 0; i < n; ++i) { xa += i; ya += y[i]; }
    xa /= n;
    ya /= n;
    double sx = 0, sxy = 0, sy = 0;
    for (uint32_t i = 0; i < n; ++i) {
        double vy = (double)y[i];
        sx += (double)((i - xa) * (i - xa));
        sxy += (double)((i - xa) * (vy - ya));
        sy += (double)((vy - ya) * (vy - ya));
    }
    (void)sy;
    float fa = (float)(sxy / sx);
    float fb = (float)(ya - fa * xa);
    float rl = 0, rr = 0;
    for (uint32_t i = 0; i < n; ++i) {
        float px = ((float)y[i] - fb) / fa;
        if (px - (float)i > rl) rl = px - (float)i;
        else if (px - (float)i < rr) rr = px - (float)i;
    }
    *a = fa;
    *b = fb;
    *L = (uint32_t)rl + 1u;
    *R = (uint32_t)(0 - rr) + 1u;
}

/* LRC_Generator.cu:221-287: double fit; float slope, int intercept (trunc),
 * float search range. */
void or_fit_lrc(const uint32_t *y, uint32_t n, float *slope, int32_t *icpt, float *range) {
    if (n == 0) { *slope = 1.0f; *icpt = 0; *range = 0.0f; return; }
    if (n == 1) { *slope = 1.0f; *icpt = (int32_t)y[0]; *range = 0.0f; return; }
    double xa = 0, ya = 0;
    for (uint32_t i = 0; i < n; ++i) { xa += i; ya += y[i]; }
    xa /= n;
    ya /= n;
    double sx = 0, sxy = 0;
    for (uint32_t i = 0; i < n; ++i) {
        double vy = (double)y[i];
        sx += (double)((i - xa) * (i - xa));
        sxy += (double)((i - xa) * (vy - ya));
    }
    double ds = sxy / sx;
    double di = ya - ds * xa;
    double rl = 0, rr = 0;
    for (uint32_t i = 0; i < n; ++i) {
        double px = (y[i] - di) / ds;
        if (px - i > rl) rl = px - i;
        else if (px - i < rr) rr = px - i;
    }
    *slope = (float)ds;
    *icpt = (int32_t)di;
    *range = (float)(rl - rr);
}

/* Predicted value of the list/segment regressions, as the reference's nvcc-
 * compiled kernels evaluate it:
 *  LRC    (LRC_Generator_kernel.cu:70, LRC_Decompression_kernel.cu:254):
 *         int((float)i * slope) + icpt — one FP32 multiply, truncated.
 *  others (SegLRC_Generator_kernel.cu:82, SegLRC_Decompression_kernel.cu:252,
 *         LRCSeg_Decompression_kernel.cu:259, HS_SegLRC_Intersection_kernel.cu:325):
 *         (int)((float)i * a + b), which nvcc contracts into one fma.rn.f32. */
#include <math.h>
/* cvt.rzi.s32.f32 (the device conversion the reference's kernels use):
 * truncation toward zero, saturating out-of-range values, NaN -> 0. */
static inline int32_t or_f2i_sat(float v) {
    if (isnan(v)) return 0;
    if (v >= 2147483648.0f) return 2147483647;
    if (v <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)v;
}
static inline int32_t or_pred_lrc(uint32_t i, float slope) {
    volatile float p = (float)(int32_t)i * slope;
    return or_f2i_sat(p);
}
static inline int32_t or_pred_fma(uint32_t i, float a, float b) { return or_f2i_sat(fmaf((float)i, a, b)); }

/* ---------------------------------------------------------------------------
 * List encoders. Each produces, for one sorted docID list, the per-segment
 * arrays of the reference's on-disk formats:
 *   words   : ParaPFD blocks of the list, concatenated
 *   off[s]  : word offset of segment s within the list (segOffset)
 *   head[s] : first docID of segment s (segHead)
 *   median  : ParaPFD only, docID at the segment's middle (segMedian)
 *   start[s]: first element index of segment s
 *   reg[s]  : {a, b, L, R} regression per segment (SegLRC/HS) as 4 u32
 *   base[s] : per-segment minimum residual (LRCSeg/SegLRC/HS)
 * ------------------------------------------------------------------------- */

/* ParaPFD_Compression/main.cpp:163-189: d-gaps across the whole list, blocks of
 * `bs`, segHead/segMedian/segOffset per block. Returns total words or -1. */
int64_t or_encode_parapfd_list(const uint32_t *docs, uint32_t n, uint32_t bs, float frac,
                               uint32_t *words, uint32_t *off, uint32_t *head, uint32_t *median) {
    if (n == 0) return -1;
    uint32_t *gaps = (uint32_t *)malloc((size_t)n * 4);
    gaps[0] = docs[0];
    for (uint32_t j = 1; j < n; ++j) gaps[j] = docs[j] - docs[j - 1];
    uint32_t nseg = (n + bs - 1) / bs;
    uint64_t nw = 0;
    for (uint32_t s = 0; s < nseg; ++s) {
        uint32_t st = s * bs;
        uint32_t cnt = (s + 1 < nseg) ? bs : n - st;
        head[s] = docs[st];
        median[s] = docs[st + cnt / 2];
        off[s] = (uint32_t)nw;
        int err;
        uint32_t w = or_parapfd_encode_block(gaps + st, cnt, frac, words + nw, &err);
        if (err) { free(gaps); return -1; }
        nw += w;
    }
    free(gaps);
    return (int64_t)nw;
}

/* NewPFD_Compression/main.cpp: the same d-gap layout with NewPFD blocks. */
int64_t or_encode_newpfd_list(const uint32_t *docs, uint32_t n, uint32_t bs, float frac,
                              uint32_t *words, uint32_t *off, uint32_t *head, uint32_t *median) {
    if (n == 0) return -1;
    uint32_t *gaps = (uint32_t *)malloc((size_t)n * 4);
    gaps[0] = docs[0];
    for (uint32_t j = 1; j < n; ++j) gaps[j] = docs[j] - docs[j - 1];
    uint32_t nseg = (n + bs - 1) / bs;
    uint64_t nw = 0;
    for (uint32_t s = 0; s < nseg; ++s) {
        uint32_t st = s * bs;
        uint32_t cnt = (s + 1 < nseg) ? bs : n - st;
        head[s] = docs[st];
        median[s] = docs[st + cnt / 2];
        off[s] = (uint32_t)nw;
        int err;
        uint32_t w = or_newpfd_encode_block(gaps + st, cnt, frac, words + nw, &err);
        if (err) { free(gaps); return -1; }
        nw += w;
    }
    free(gaps);
    return (int64_t)nw;
}

/* Same d-gap encoding with explicit segment starts (hash-bucketed lists:
 * blocks never cross a bucket boundary). */
int64_t or_encode_parapfd_segs(const uint32_t *docs, uint32_t n, uint32_t nseg, const uint32_t *start, float frac,
                               uint32_t *words, uint32_t *off, uint32_t *head, uint32_t *median) {
    if (n == 0 || nseg == 0) return -1;
    uint32_t *gaps = (uint32_t *)malloc((size_t)n * 4);
    gaps[0] = docs[0];
    for (uint32_t j = 1; j < n; ++j) gaps[j] = docs[j] - docs[j - 1];
    uint64_t nw = 0;
    for (uint32_t s = 0; s < nseg; ++s) {
        uint32_t st = start[s];
        uint32_t cnt = ((s + 1 < nseg) ? start[s + 1] : n) - st;
        head[s] = docs[st];
        median[s] = docs[st + cnt / 2];
        off[s] = (uint32_t)nw;
        int err;
        uint32_t w = or_parapfd_encode_block(gaps + st, cnt, frac, words + nw, &err);
        if (err) { free(gaps); return -1; }
        nw += w;
    }
    free(gaps);
    return (int64_t)nw;
}

/* Residual encoders share the block layout: the residual array is cut into
 * segments (fixed `bs`, or the given `start` boundaries for HS) and each
 * segment is one ParaPFD block. `codec`: 1 LRC, 2 LRCSeg, 3 SegLRC, 4 HS_SegLRC.
 * listreg receives the list-level regression: LRC {slope, icpt, range, 0};
 * LRCSeg/SegLRC {a, b, L, R} (as raw u32 bit patterns).
 * LRC_Generator.cu:155-178 (LRC residual, min folded into the intercept);
 * LRCSeg_Generator_kernel.cu:62-101 + LRCSeg_Generator.cu:185-230 (list
 * regression, per-segment base); SegLRC_Generator.cu:181-229 + kernel :62-103
 * (per-segment regression and base); HS_SegLRC_Generator.cu:95-288 (per-bucket
 * regression and base; the element's own bucket is used, as the reference
 * decoder HS_SegLRC_Intersection_kernel.cu:279-325 reads it). */
int64_t or_encode_residual_list(int codec, const uint32_t *docs, uint32_t n, uint32_t nseg,
                                const uint32_t *start, float frac,
                                uint32_t *words, uint32_t *off, uint32_t *head,
                                uint32_t *reg, int32_t *base, uint32_t *listreg) {
    if (n == 0 || nseg == 0) return -1;
    int32_t *res = (int32_t *)malloc((size_t)n * 4);
    if (codec == 1) {
        float slope, range;
        int32_t icpt;
        or_fit_lrc(docs, n, &slope, &icpt, &range);
        if (n > 1) {
            for (uint32_t i = 0; i < n; ++i) {
                int32_t y = (int32_t)((uint32_t)or_pred_lrc(i, slope) + (uint32_t)icpt);
                res[i] = (int32_t)(docs[i] - (uint32_t)y);
            }
            int32_t mn = res[0];
            for (uint32_t i = 1; i < n; ++i) if (res[i] < mn) mn = res[i];
            for (uint32_t i = 0; i < n; ++i) res[i] -= mn;
            icpt = (int32_t)((uint32_t)icpt + (uint32_t)mn);
        } else {
            res[0] = 0;
        }
        memcpy(&listreg[0], &slope, 4);
        memcpy(&listreg[1], &icpt, 4);
        memcpy(&listreg[2], &range, 4);
        listreg[3] = 0;
    } else {
        float la, lb;
        uint32_t lL, lR;
        or_fit_seg(docs, n, &la, &lb, &lL, &lR);
        memcpy(&listreg[0], &la, 4);
        memcpy(&listreg[1], &lb, 4);
        listreg[2] = lL;
        listreg[3] = lR;
        for (uint32_t s = 0; s < nseg; ++s) {
            uint32_t st = start[s], en = (s + 1 < nseg) ? start[s + 1] : n;
            float a = la, b = lb;
            if (codec != 2) {
                uint32_t L, R;
                or_fit_seg(docs + st, en - st, &a, &b, &L, &R);
                memcpy(&reg[4 * s + 0], &a, 4);
                memcpy(&reg[4 * s + 1], &b, 4);
                reg[4 * s + 2] = L;
                reg[4 * s + 3] = R;
            }
            for (uint32_t i = st; i < en; ++i) {
                uint32_t idx = (codec == 2) ? i : i - st;
                int32_t y = or_pred_fma(idx, a, b);
                res[i] = (int32_t)(docs[i] - (uint32_t)y);
            }
            int32_t mn = res[st];
            for (uint32_t i = st + 1; i < en; ++i) if (res[i] < mn) mn = res[i];
            for (uint32_t i = st; i < en; ++i) {
                int64_t r = (int64_t)res[i] - (int64_t)mn;
                if (r > 0x7fffffffLL) { free(res); return -1; }
                res[i] = (int32_t)r;
            }
            base[s] = mn;
        }
    }
    uint64_t nw = 0;
    for (uint32_t s = 0; s < nseg; ++s) {
        uint32_t st = start[s], en = (s + 1 < nseg) ? start[s + 1] : n;
        head[s] = docs[st];
        off[s] = (uint32_t)nw;
        int err;
        uint32_t w = or_parapfd_encode_block((const uint32_t *)res + st, en - st, frac, words + nw, &err);
        if (err) { free(res); return -1; }
        nw += w;
    }
    free(res);
    return (int64_t)nw;
}

/* HS_SegLRC_Generator.cu:503-594 (RunGetHashInfo): shift from the list length
 * (expected bucket size `ebs`), or a fixed number of top bits `kbits` of a
 * `ubits`-bit universe when kbits > 0. Writes bucket boundaries bnd[0..nb]
 * (bnd[b] = first element whose docID >> shift >= b) and returns nb; *shift out. */
uint32_t or_hs_partition(const uint32_t *docs, uint32_t n, uint32_t ebs, uint32_t kbits, uint32_t ubits,
                         uint32_t *shift_out, uint32_t *bnd) {
    uint32_t maxbits = or_bits(docs[n - 1]);
    uint32_t shift;
    if (kbits > 0) {
        shift = ubits > kbits ? ubits - kbits : 0;
    } else if (n <= ebs) {
        *shift_out = maxbits;
        bnd[0] = 0;
        bnd[1] = n;
        return 1;
    } else {
        uint32_t expected = (n + ebs - 1) / ebs;
        shift = maxbits - or_bits(expected);
    }
    *shift_out = shift;
    uint32_t cur = 0;
    bnd[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t b = (shift >= 32) ? 0 : (docs[i] >> shift);
        while (cur < b) { ++cur; bnd[cur] = i; }
    }
    ++cur;
    bnd[cur] = n;
    return cur;
}

/* ---------------------------------------------------------------------------
 * Decoders of one list in the layouts above (exact, scalar).
 * ------------------------------------------------------------------------- */
int or_decode_list(int codec, const uint32_t *words, uint32_t n, uint32_t nseg, const uint32_t *start,
                   const uint32_t *off, const uint32_t *head, const uint32_t *reg, const int32_t *base,
                   const uint32_t *listreg, uint32_t *out) {
    for (uint32_t s = 0; s < nseg; ++s) {
        uint32_t st = start[s], en = (s + 1 < nseg) ? start[s + 1] : n;
        uint32_t cnt = en - st;
        if (codec == 6) or_newpfd_decode_block(words + off[s], cnt, out + st);
        else or_parapfd_decode_block(words + off[s], cnt, out + st);
        if (codec == 0 || codec == 6) {
            /* ParaPFD_Decompression_kernel.cu:244-263: element 0 := segHead, scan */
            out[st] = head[s];
            for (uint32_t i = st + 1; i < en; ++i) out[i] += out[i - 1];
        } else if (codec == 1) {
            float slope; int32_t icpt;
            memcpy(&slope, &listreg[0], 4);
            memcpy(&icpt, &listreg[1], 4);
            for (uint32_t i = st; i < en; ++i) out[i] += (uint32_t)or_pred_lrc(i, slope) + (uint32_t)icpt;
        } else {
            float a, b;
            if (codec == 2) { memcpy(&a, &listreg[0], 4); memcpy(&b, &listreg[1], 4); }
            else { memcpy(&a, &reg[4 * s], 4); memcpy(&b, &reg[4 * s + 1], 4); }
            for (uint32_t i = st; i < en; ++i) {
                uint32_t idx = (codec == 2) ? i : i - st;
                out[i] += (uint32_t)or_pred_fma(idx, a, b) + (uint32_t)base[s];
            }
        }
    }
    return OR_OK;
}

/* ---------------------------------------------------------------------------
 * Exact intersection of sorted lists, and the reference's checksum triple.
 * ------------------------------------------------------------------------- */

/* galloping lower bound: first index >= lo with a[idx] >= key */
static uint64_t or_gallop(const uint32_t *a, uint64_t lo, uint64_t n, uint32_t key) {
    uint64_t step = 1, hi = lo;
    while (hi < n && a[hi] < key) { lo = hi + 1; hi += step; step <<= 1; }
    if (hi > n) hi = n;
    while (lo < hi) {
        uint64_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

/* Exact AND of k sorted lists (any order); writes the sorted result, returns count. */
uint64_t or_intersect(uint32_t k, const uint32_t *const *lists, const uint64_t *lens, uint32_t *out) {
    if (k == 0) return 0;
    uint32_t sh = 0;
    for (uint32_t j = 1; j < k; ++j) if (lens[j] < lens[sh]) sh = j;
    uint64_t *cur = (uint64_t *)calloc(k, sizeof(uint64_t));
    uint64_t r = 0;
    for (uint64_t i = 0; i < lens[sh]; ++i) {
        uint32_t key = lists[sh][i];
        int ok = 1;
        for (uint32_t j = 0; j < k && ok; ++j) {
            if (j == sh) continue;
            cur[j] = or_gallop(lists[j], cur[j], lens[j], key);
            if (cur[j] >= lens[j] || lists[j][cur[j]] != key) ok = 0;
        }
        if (ok) out[r++] = key;
    }
    free(cur);
    return r;
}

/* ParaPFD_Intersection.cu:378-403 (verify) with ParaPFD_Intersection_kernel.cu:78-82:
 * cs[0] = #queries with empty result, cs[1] = total results, cs[2] = XOR over
 * non-empty queries of result[0] ^ result[n-1] ^ result[n/2]. */
void or_checksum(uint32_t nq, const uint64_t *offsets, const uint32_t *res, uint64_t *cs) {
    for (uint32_t q = 0; q < nq; ++q) {
        uint64_t n = offsets[q + 1] - offsets[q];
        if (n) {
            const uint32_t *r = res + offsets[q];
            cs[1] += n;
            cs[2] ^= r[0];
            cs[2] ^= r[n - 1];
            cs[2] ^= r[n / 2];
        } else {
            ++cs[0];
        }
    }
}

/* ---------------------------------------------------------------------------
 * Learned position model (no reference counterpart; checks the library's
 * training kernels and its exactness claim). Parameter layout:
 * w1[32] b1[32] w2[32][32] b2[32] w3[32] b3.
 * ------------------------------------------------------------------------- */
#define OR_H 32
#define OR_NP (OR_H + OR_H + OR_H * OR_H + OR_H + OR_H + 1)

/* Gradient of mean((f(x) - y)^2) in double precision. */
void or_mlp_grad(const float *P, const float *x, const float *y, uint32_t n, double *grad, double *loss) {
    const float *w1 = P, *b1 = P + OR_H, *w2 = P + 2 * OR_H, *b2 = w2 + OR_H * OR_H, *w3 = b2 + OR_H, *b3 = w3 + OR_H;
    for (int j = 0; j < OR_NP; ++j) grad[j] = 0;
    double L = 0;
    for (uint32_t s = 0; s < n; ++s) {
        double z1[OR_H], h1[OR_H], z2[OR_H], h2[OR_H];
        for (int i = 0; i < OR_H; ++i) { z1[i] = (double)w1[i] * x[s] + b1[i]; h1[i] = z1[i] > 0 ? z1[i] : 0; }
        double out = b3[0];
        for (int o = 0; o < OR_H; ++o) {
            double acc = b2[o];
            for (int i = 0; i < OR_H; ++i) acc += (double)w2[o * OR_H + i] * h1[i];
            z2[o] = acc;
            h2[o] = acc > 0 ? acc : 0;
            out += (double)w3[o] * h2[o];
        }
        const double d = out - y[s];
        L += d * d;
        const double dout = 2.0 * d / n;
        double dz2[OR_H];
        for (int o = 0; o < OR_H; ++o) {
            grad[2 * OR_H + OR_H * OR_H + OR_H + o] += dout * h2[o];  /* w3 */
            dz2[o] = z2[o] > 0 ? dout * w3[o] : 0;
            grad[2 * OR_H + OR_H * OR_H + o] += dz2[o];               /* b2 */
            for (int i = 0; i < OR_H; ++i) grad[2 * OR_H + o * OR_H + i] += dz2[o] * h1[i];
        }
        grad[OR_NP - 1] += dout;                                        /* b3 */
        for (int i = 0; i < OR_H; ++i) {
            double dh = 0;
            for (int o = 0; o < OR_H; ++o) dh += (double)w2[o * OR_H + i] * dz2[o];
            const double dz1 = z1[i] > 0 ? dh : 0;
            grad[i] += dz1 * x[s];                                      /* w1 */
            grad[OR_H + i] += dz1;                                      /* b1 */
        }
    }
    *loss = L / n;
}

/* The query-time inference in single precision, operation for operation as
 * the device evaluates it (fused multiply-adds in the same order). */
static float or_mlp_root(const float *P, float x) {
    const float *w1 = P, *b1 = P + OR_H, *w2 = P + 2 * OR_H, *b2 = w2 + OR_H * OR_H, *w3 = b2 + OR_H, *b3 = w3 + OR_H;
    float h1[OR_H];
    for (int i = 0; i < OR_H; ++i) h1[i] = fmaxf(fmaf(w1[i], x, b1[i]), 0.0f);
    float out = b3[0];
    for (int o = 0; o < OR_H; ++o) {
        float acc = b2[o];
        for (int i = 0; i < OR_H; ++i) acc = fmaf(w2[o * OR_H + i], h1[i], acc);
        out = fmaf(w3[o], fmaxf(acc, 0.0f), out);
    }
    return out;
}

/* Leaf of each key as the network routes it (single-precision restatement). */
void or_model_leaves(const float *P, float kmin, float kscale, uint32_t nleaves, const uint32_t *keys, uint64_t n,
                     uint32_t *out) {
    for (uint64_t p = 0; p < n; ++p) {
        volatile float xs = (float)keys[p] - kmin;
        const float x = xs * kscale;
        volatile float f = or_mlp_root(P, x) * (float)nleaves;
        int li = (int)floorf(f);
        if (li < 0) li = 0;
        if (li >= (int)nleaves) li = (int)nleaves - 1;
        out[p] = (uint32_t)li;
    }
}

/* For every key of a sorted list: its leaf and whether its rank lies inside
 * the leaf's window. leaves: 4 x 32-bit per leaf {a, b, elo, ehi}. Returns the
 * number of keys outside their window (0 when the model is exact) and fills
 * per-leaf key counts if counts != NULL. */
uint64_t or_model_check(const float *P, float kmin, float kscale, uint32_t nleaves, const int32_t *leaves,
                        const uint32_t *keys, uint64_t n, uint32_t *counts) {
    uint64_t bad = 0;
    for (uint64_t p = 0; p < n; ++p) {
        volatile float xs = (float)keys[p] - kmin;
        const float x = xs * kscale;
        const float r = or_mlp_root(P, x);
        volatile float f = r * (float)nleaves;
        int li = (int)floorf(f);
        if (li < 0) li = 0;
        if (li >= (int)nleaves) li = (int)nleaves - 1;
        float a, b;
        memcpy(&a, &leaves[4 * li], 4);
        memcpy(&b, &leaves[4 * li + 1], 4);
        float pr = fmaf(a, x, b);
        pr = fminf(fmaxf(pr, -1.0e9f), 1.0e9f);
        const int64_t pred = (int64_t)floorf(pr);
        const int64_t lo = pred + leaves[4 * li + 2], hi = pred + leaves[4 * li + 3];
        if ((int64_t)p < lo || (int64_t)p > hi) ++bad;
        if (counts) ++counts[li];
    }
    return bad;
}

/* ---------------------------------------------------------------------------
 * CPU path over the compressed index image (the layout libexcl_gpu exports:
 * per list {codec, n, seg_base, nseg, word_base, reg[4]}, per segment head,
 * rec {start, off, aux, count}, reg {a, b, L, R}). Per query: decode the
 * shortest list; for each longer list walk its segment heads with a cursor
 * (keys ascend), decode a segment once when a key first lands in it
 * (ParaPFor.cpp decodeBlock + the codec's reconstruction) and binary-search
 * the key there. This is the reference's decode + AND on the host.
 * ------------------------------------------------------------------------- */
typedef struct {
    const uint32_t *words;
    const uint32_t *lcodec, *ln, *lseg, *lnseg;
    const uint64_t *lword;
    const uint32_t *lreg;     /* 4 per list */
    const uint32_t *head;
    const uint32_t *rec;      /* 4 per segment */
    const uint32_t *sreg;     /* 4 per segment */
} or_image;

static void or_decode_seg(const or_image *im, uint32_t l, uint32_t s, uint32_t *out) {
    const uint32_t sg = im->lseg[l] + s;
    const uint32_t *r = im->rec + 4 * (size_t)sg;
    const uint32_t st = r[0], cnt = r[3];
    const uint32_t codec = im->lcodec[l];
    if (codec == 6) or_newpfd_decode_block(im->words + im->lword[l] + r[1], cnt, out);
    else or_parapfd_decode_block(im->words + im->lword[l] + r[1], cnt, out);
    if (codec == 0 || codec == 5 || codec == 6) {
        out[0] = im->head[sg];
        for (uint32_t i = 1; i < cnt; ++i) out[i] += out[i - 1];
    } else if (codec == 1) {
        float slope; int32_t icpt;
        memcpy(&slope, &im->lreg[4 * l], 4);
        memcpy(&icpt, &im->lreg[4 * l + 1], 4);
        for (uint32_t i = 0; i < cnt; ++i) out[i] += (uint32_t)or_pred_lrc(st + i, slope) + (uint32_t)icpt;
    } else {
        float a, b;
        if (codec == 2) { memcpy(&a, &im->lreg[4 * l], 4); memcpy(&b, &im->lreg[4 * l + 1], 4); }
        else { memcpy(&a, &im->sreg[4 * (size_t)sg], 4); memcpy(&b, &im->sreg[4 * (size_t)sg + 1], 4); }
        for (uint32_t i = 0; i < cnt; ++i) {
            uint32_t idx = (codec == 2) ? st + i : i;
            out[i] += (uint32_t)or_pred_fma(idx, a, b) + r[2];
        }
    }
}

typedef struct {
    const or_image *im;
    const uint32_t *terms;
    const uint64_t *toff;
    uint32_t q0, q1;
    uint64_t *counts;
    uint32_t *keys, *tmp, *seg;
} or_cjob;

static void *or_cworker(void *arg) {
    or_cjob *j = (or_cjob *)arg;
    const or_image *im = j->im;
    for (uint32_t q = j->q0; q < j->q1; ++q) {
        uint32_t k = (uint32_t)(j->toff[q + 1] - j->toff[q]);
        const uint32_t *t = j->terms + j->toff[q];
        if (k == 0) { j->counts[q] = 0; continue; }
        uint32_t sh = 0;
        for (uint32_t i = 1; i < k; ++i) if (im->ln[t[i]] < im->ln[t[sh]]) sh = i;
        /* decode the shortest list */
        uint32_t ls = t[sh], n = 0;
        for (uint32_t s = 0; s < im->lnseg[ls]; ++s) {
            or_decode_seg(im, ls, s, j->keys + n);
            n += im->rec[4 * (size_t)(im->lseg[ls] + s) + 3];
        }
        /* probe the others in ascending length */
        uint8_t done[64] = {0};
        done[sh] = 1;
        for (uint32_t r = 1; r < k && n; ++r) {
            uint32_t b = 0;
            while (done[b]) ++b;
            for (uint32_t i = b + 1; i < k; ++i) if (!done[i] && im->ln[t[i]] < im->ln[t[b]]) b = i;
            done[b] = 1;
            const uint32_t l = t[b];
            const uint32_t *hd = im->head + im->lseg[l];
            const uint32_t ns = im->lnseg[l];
            uint32_t cur = 0, cached = 0xffffffffu, cnt = 0, m = 0;
            for (uint32_t i = 0; i < n; ++i) {
                const uint32_t key = j->keys[i];
                if (key < hd[0]) continue;
                /* gallop to the last head <= key */
                uint32_t step = 1, hi = cur + 1;
                while (hi < ns && hd[hi] <= key) { cur = hi; hi += step; step <<= 1; }
                if (hi > ns) hi = ns;
                uint32_t lo = cur;
                while (lo + 1 < hi) { uint32_t mid = (lo + hi) >> 1; if (hd[mid] <= key) lo = mid; else hi = mid; }
                cur = lo;
                if (cur != cached) {
                    or_decode_seg(im, l, cur, j->seg);
                    cnt = im->rec[4 * (size_t)(im->lseg[l] + cur) + 3];
                    cached = cur;
                }
                uint32_t a = 0, z = cnt;
                while (a < z) { uint32_t mid = (a + z) >> 1; if (j->seg[mid] < key) a = mid + 1; else z = mid; }
                if (a < cnt && j->seg[a] == key) j->keys[m++] = key;
            }
            n = m;
        }
        j->counts[q] = n;
    }
    return NULL;
}

/* Runs queries [0, nq) over the compressed image on `threads` threads; wall seconds. */
double or_run_queries_compressed(const uint32_t *words, const uint32_t *lcodec, const uint32_t *ln,
                                 const uint32_t *lseg, const uint32_t *lnseg, const uint64_t *lword,
                                 const uint32_t *lreg, const uint32_t *head, const uint32_t *rec,
                                 const uint32_t *sreg, const uint32_t *terms, const uint64_t *toff, uint32_t nq,
                                 uint32_t threads, uint32_t max_list, uint32_t max_seg, uint64_t *counts) {
    or_image im = {words, lcodec, ln, lseg, lnseg, lword, lreg, head, rec, sreg};
    if (threads < 1) threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    or_cjob *jobs = (or_cjob *)malloc(sizeof(or_cjob) * threads);
    for (uint32_t t = 0; t < threads; ++t) {
        jobs[t].im = &im; jobs[t].terms = terms; jobs[t].toff = toff;
        jobs[t].q0 = (uint32_t)((uint64_t)nq * t / threads);
        jobs[t].q1 = (uint32_t)((uint64_t)nq * (t + 1) / threads);
        jobs[t].counts = counts;
        jobs[t].keys = (uint32_t *)malloc(((size_t)max_list + 8) * 4);
        jobs[t].seg = (uint32_t *)malloc(((size_t)max_seg + 8) * 4);
        jobs[t].tmp = NULL;
    }
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    for (uint32_t t = 0; t < threads; ++t) pthread_create(&th[t], NULL, or_cworker, &jobs[t]);
    for (uint32_t t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    clock_gettime(CLOCK_MONOTONIC, &b);
    for (uint32_t t = 0; t < threads; ++t) { free(jobs[t].keys); free(jobs[t].seg); }
    free(th);
    free(jobs);
    return (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
}

/* ---------------------------------------------------------------------------
 * Threaded CPU baseline over already-decoded lists (CSR): per query, exact
 * galloping AND.
 * ------------------------------------------------------------------------- */
typedef struct {
    const uint32_t *docs;
    const uint64_t *loff;
    const uint32_t *terms;
    const uint64_t *toff;
    uint32_t q0, q1;
    uint64_t *counts;
    uint32_t *scratch;
} or_job;

static void *or_worker(void *arg) {
    or_job *j = (or_job *)arg;
    const uint32_t *lp[64];
    uint64_t ln[64];
    for (uint32_t q = j->q0; q < j->q1; ++q) {
        uint64_t t0 = j->toff[q], t1 = j->toff[q + 1];
        uint32_t k = (uint32_t)(t1 - t0);
        if (k > 64) k = 64;
        for (uint32_t t = 0; t < k; ++t) {
            uint32_t term = j->terms[t0 + t];
            lp[t] = j->docs + j->loff[term];
            ln[t] = j->loff[term + 1] - j->loff[term];
        }
        j->counts[q] = or_intersect(k, lp, ln, j->scratch);
    }
    return NULL;
}

/* Runs all queries on `threads` threads, returns wall seconds; counts[q] out. */
double or_run_queries(const uint32_t *docs, const uint64_t *loff, const uint32_t *terms, const uint64_t *toff,
                      uint32_t nq, uint32_t threads, uint64_t max_list, uint64_t *counts) {
    if (threads < 1) threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    or_job *jobs = (or_job *)malloc(sizeof(or_job) * threads);
    struct timespec a, b;
    for (uint32_t t = 0; t < threads; ++t) {
        jobs[t].docs = docs; jobs[t].loff = loff; jobs[t].terms = terms; jobs[t].toff = toff;
        jobs[t].q0 = (uint32_t)((uint64_t)nq * t / threads);
        jobs[t].q1 = (uint32_t)((uint64_t)nq * (t + 1) / threads);
        jobs[t].counts = counts;
        jobs[t].scratch = (uint32_t *)malloc((max_list ? max_list : 1) * 4);
    }
    clock_gettime(CLOCK_MONOTONIC, &a);
    for (uint32_t t = 0; t < threads; ++t) pthread_create(&th[t], NULL, or_worker, &jobs[t]);
    for (uint32_t t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    clock_gettime(CLOCK_MONOTONIC, &b);
    for (uint32_t t = 0; t < threads; ++t) free(jobs[t].scratch);
    free(th);
    free(jobs);
    return (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
}
