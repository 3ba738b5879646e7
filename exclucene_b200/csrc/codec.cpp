// Host side of the index: ParaPFD block codec, regression fits, hash-segment
// partitioning and the index builder that lays a set of sorted docID lists out
// as the device-resident image (words + per-list + per-segment arrays).
//
// Bit-exactness notes
//  * Block bytes follow ParaPFor.cpp:56-126 (descriptor lb<<26|eb<<21|hb<<16|en,
//    LSB-first packing of lows, exception positions, exception high bits).
//  * The regression fits follow the reference's double-precision host code
//    (SegLRC_Generator.cu:264-331, LRC_Generator.cu:221-287). This file is
//    compiled with -ffp-contract=off and no -march flag so that, like the
//    reference host compiler, no multiply-add is fused.
//  * The predicted values follow the reference's device code: LRC truncates a
//    single FP32 product (LRC_Generator_kernel.cu:70); LRCSeg, SegLRC and HS
//    evaluate (int)(i*a+b), which nvcc contracts into one fma.rn.f32
//    (SegLRC_Generator_kernel.cu:82) — std::fmaf is that same correctly
//    rounded operation.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>

#include "excl_internal.h"

namespace excl {

static inline uint32_t nbits(uint32_t v) { return v ? 32u - (uint32_t)__builtin_clz(v) : 0u; }
static inline uint64_t words_for(uint64_t nvals, uint32_t bits) { return (nvals * bits + 31u) >> 5; }

// Streams `bits`-bit values LSB-first into out[] (which it zero-fills).
static void pack_bits(const uint32_t *v, uint32_t n, uint32_t bits, uint32_t *out) {
    uint64_t nw = words_for(n, bits);
    if (bits == 0) return;
    uint64_t acc = 0;
    uint32_t fill = 0;
    uint64_t w = 0;
    for (uint32_t i = 0; i < n; ++i) {
        acc |= (uint64_t)v[i] << fill;
        fill += bits;
        while (fill >= 32) {
            out[w++] = (uint32_t)acc;
            acc >>= 32;
            fill -= 32;
        }
    }
    if (fill) out[w++] = (uint32_t)acc;
    for (; w < nw; ++w) out[w] = 0;
}

static void unpack_bits(const uint32_t *in, uint32_t n, uint32_t bits, uint32_t *out) {
    if (bits == 0) {
        std::fill(out, out + n, 0u);
        return;
    }
    const uint64_t mask = (bits >= 32) ? 0xffffffffull : ((1ull << bits) - 1);
    uint64_t acc = 0;
    uint32_t have = 0;
    uint64_t r = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (have < bits) {
            acc |= (uint64_t)in[r++] << have;
            have += 32;
        }
        out[i] = (uint32_t)(acc & mask);
        acc >>= bits;
        have -= bits;
    }
}

// Smallest b with #(v >= 2^b) satisfying (float)nEx <= frac * n in single
// precision (ParaPFor.cpp:31-53), computed from a histogram of bit lengths.
static uint32_t best_b(const uint32_t *in, uint32_t n, float frac) {
    uint32_t hist[33] = {0};
    for (uint32_t i = 0; i < n; ++i) ++hist[nbits(in[i])];
    // values with nbits(v) > b are exceptions for width b
    uint32_t above = n - hist[0];
    for (uint32_t b = 0; b < 32; ++b) {
        if ((float)above <= frac * (float)n) return b;
        above -= hist[b + 1];
    }
    return 32;
}

// ---------------------------------------------------------------------------
// NewPFD blocks (NewPFor.cpp:52-139): descriptor b << 26 | en, the b-bit low
// parts, then one Simple-16 stream holding the exception positions (first
// absolute, then gaps minus one) followed by their high parts.

// Simple-16 word layouts (Zhang, Long and Suel, WWW 2008; the same 16 cases as
// the reference's Simple16.h): a 4-bit selector and 28 data bits split into the
// listed runs of equal widths, low bits first.
struct S16Run {
    uint8_t count, width;
};
static const S16Run kS16Runs[16][3] = {
    {{28, 1}, {0, 0}, {0, 0}}, {{7, 2}, {14, 1}, {0, 0}}, {{7, 1}, {7, 2}, {7, 1}}, {{14, 1}, {7, 2}, {0, 0}},
    {{14, 2}, {0, 0}, {0, 0}}, {{1, 4}, {8, 3}, {0, 0}},  {{1, 3}, {4, 4}, {3, 3}}, {{7, 4}, {0, 0}, {0, 0}},
    {{4, 5}, {2, 4}, {0, 0}},  {{2, 4}, {4, 5}, {0, 0}},  {{3, 6}, {2, 5}, {0, 0}}, {{2, 5}, {3, 6}, {0, 0}},
    {{4, 7}, {0, 0}, {0, 0}},  {{1, 10}, {2, 9}, {0, 0}}, {{2, 14}, {0, 0}, {0, 0}}, {{1, 28}, {0, 0}, {0, 0}},
};

struct S16Table {
    uint8_t count[16];
    uint8_t width[16][28];
    S16Table() {
        for (int k = 0; k < 16; ++k) {
            int c = 0, bits = 0;
            for (const S16Run &r : kS16Runs[k])
                for (int j = 0; j < r.count; ++j, ++c) {
                    width[k][c] = r.width;
                    bits += r.width;
                }
            count[k] = (uint8_t)c;
            if (bits != 28) std::abort();  // every layout fills the 28 data bits
        }
    }
};
static const S16Table &s16() {
    static const S16Table t;
    return t;
}

// Appends v[0..n) as Simple-16 words: each word takes the first layout whose
// widths hold the next min(count, left) values. False if a value needs more
// than 28 bits (no layout holds it).
static bool s16_encode(const uint32_t *v, uint32_t n, std::vector<uint32_t> &out) {
    const S16Table &t = s16();
    uint32_t i = 0;
    while (i < n) {
        bool done = false;
        for (int k = 0; k < 16 && !done; ++k) {
            const uint32_t vol = std::min<uint32_t>(t.count[k], n - i);
            uint32_t j = 0;
            while (j < vol && (uint64_t)v[i + j] < (1ull << t.width[k][j])) ++j;
            if (j < vol) continue;
            uint32_t w = (uint32_t)k << 28, sh = 0;
            for (j = 0; j < vol; ++j) {
                w |= v[i + j] << sh;
                sh += t.width[k][j];
            }
            out.push_back(w);
            i += vol;
            done = true;
        }
        if (!done) return false;
    }
    return true;
}

// Decodes Simple-16 words from `in` until n values are out; returns words read.
static uint32_t s16_decode(const uint32_t *in, uint32_t n, uint32_t *out) {
    const S16Table &t = s16();
    uint32_t r = 0, i = 0;
    while (i < n) {
        const uint32_t w = in[r++], k = w >> 28;
        uint32_t sh = 0;
        for (uint32_t j = 0; j < t.count[k] && i < n; ++j) {
            out[i++] = (w >> sh) & ((1u << t.width[k][j]) - 1u);
            sh += t.width[k][j];
        }
    }
    return r;
}

uint32_t newpfd_encode_block(const uint32_t *in, uint32_t n, float frac, uint32_t *out, int *err);
uint32_t newpfd_decode_block(const uint32_t *in, uint32_t n, uint32_t *out);

uint32_t pfd_encode_block(const uint32_t *in, uint32_t n, float frac, uint32_t *out, int *err) {
    *err = EXCL_OK;
    const uint32_t lb = best_b(in, n, frac);
    if (lb >= 32) {
        *err = EXCL_E_FORMAT;
        return 0;
    }
    std::vector<uint32_t> low(n), pos, high;
    const uint32_t lim = 1u << lb;
    for (uint32_t i = 0; i < n; ++i) {
        if (in[i] >= lim) {
            low[i] = in[i] & (lim - 1);
            pos.push_back(i);
            high.push_back(in[i] >> lb);
        } else {
            low[i] = in[i];
        }
    }
    const uint32_t en = (uint32_t)pos.size();
    uint32_t w = 1;
    pack_bits(low.data(), n, lb, out + w);
    w += (uint32_t)words_for(n, lb);
    if (en == 0) {
        out[0] = lb << 26;
        return w;
    }
    if (en > 65535u) {
        *err = EXCL_E_FORMAT;
        return 0;
    }
    uint32_t orh = 0;
    for (uint32_t h : high) orh |= h;
    const uint32_t eb = nbits(pos.back()), hb = nbits(orh);
    if (eb >= 32 || hb >= 32) {
        *err = EXCL_E_FORMAT;
        return 0;
    }
    pack_bits(pos.data(), en, eb, out + w);
    w += (uint32_t)words_for(en, eb);
    pack_bits(high.data(), en, hb, out + w);
    w += (uint32_t)words_for(en, hb);
    out[0] = (lb << 26) + (eb << 21) + (hb << 16) + en;
    return w;
}

uint32_t newpfd_encode_block(const uint32_t *in, uint32_t n, float frac, uint32_t *out, int *err) {
    *err = EXCL_OK;
    const uint32_t b = best_b(in, n, frac);
    if (b >= 32) {
        *err = EXCL_E_FORMAT;
        return 0;
    }
    std::vector<uint32_t> low(n), pos, high;
    const uint32_t lim = 1u << b;
    for (uint32_t i = 0; i < n; ++i) {
        low[i] = in[i] & (lim - 1u);
        if (in[i] >= lim) {
            pos.push_back(i);
            high.push_back(in[i] >> b);
        }
    }
    const uint32_t en = (uint32_t)pos.size();
    if (en > 65535u) {
        *err = EXCL_E_FORMAT;
        return 0;
    }
    uint32_t w = 1;
    pack_bits(low.data(), n, b, out + w);
    w += (uint32_t)words_for(n, b);
    out[0] = (b << 26) + en;
    if (en == 0) return w;
    // positions as gaps minus one after the first, then the high parts
    std::vector<uint32_t> all(2 * (size_t)en), s16w;
    for (uint32_t i = 0; i < en; ++i) {
        all[i] = i ? pos[i] - pos[i - 1] - 1 : pos[0];
        all[en + i] = high[i];
    }
    if (!s16_encode(all.data(), 2 * en, s16w)) {
        *err = EXCL_E_FORMAT;  // an exception high part of more than 28 bits
        return 0;
    }
    std::memcpy(out + w, s16w.data(), s16w.size() * 4);
    return w + (uint32_t)s16w.size();
}

uint32_t newpfd_decode_block(const uint32_t *in, uint32_t n, uint32_t *out) {
    const uint32_t b = (in[0] >> 26) & 31u, en = in[0] & 0xffffu;
    uint32_t w = 1;
    unpack_bits(in + w, n, b, out);
    w += (uint32_t)words_for(n, b);
    if (en) {
        std::vector<uint32_t> all(2 * (size_t)en);
        w += s16_decode(in + w, 2 * en, all.data());
        uint32_t p = all[0];
        for (uint32_t i = 0; i < en; ++i) {
            if (i) p += all[i] + 1;
            if (p < n) out[p] += all[en + i] << b;
        }
    }
    return w;
}

uint64_t newpfd_block_words(const uint32_t *in, uint32_t n, uint64_t avail) {
    if (avail == 0) return ~0ull;
    const uint32_t b = (in[0] >> 26) & 31u, en = in[0] & 0xffffu;
    uint64_t w = 1 + words_for(n, b);
    if (en) {
        // count the Simple-16 words that hold 2 * en values, never reading past avail
        const S16Table &t = s16();
        uint32_t got = 0;
        while (got < 2 * en) {
            if (w >= avail) return ~0ull;
            got += t.count[in[w++] >> 28];
        }
    }
    return w <= avail ? w : ~0ull;
}

uint32_t pfd_block_words(const uint32_t *in, uint32_t n) {
    const uint32_t d = in[0];
    const uint32_t lb = (d >> 26) & 31u, eb = (d >> 21) & 31u, hb = (d >> 16) & 31u, en = d & 0xffffu;
    uint64_t w = 1 + words_for(n, lb);
    if (en) w += words_for(en, eb) + words_for(en, hb);
    return (uint32_t)w;
}

uint32_t pfd_decode_block(const uint32_t *in, uint32_t n, uint32_t *out) {
    const uint32_t d = in[0];
    const uint32_t lb = (d >> 26) & 31u, eb = (d >> 21) & 31u, hb = (d >> 16) & 31u, en = d & 0xffffu;
    uint32_t w = 1;
    unpack_bits(in + w, n, lb, out);
    w += (uint32_t)words_for(n, lb);
    if (en) {
        std::vector<uint32_t> pos(en), high(en);
        unpack_bits(in + w, en, eb, pos.data());
        w += (uint32_t)words_for(en, eb);
        unpack_bits(in + w, en, hb, high.data());
        w += (uint32_t)words_for(en, hb);
        for (uint32_t i = 0; i < en; ++i)
            if (pos[i] < n) out[pos[i]] |= high[i] << lb;
    }
    return w;
}


// ---------------------------------------------------------------------------
// Regression fits (reference host arithmetic, see header comment).

struct Fit {
    float a = 1.0f, b = 0.0f;
    uint32_t L = 0, R = 0;
};

static Fit fit_segment(const uint32_t *y, uint32_t n) {
    Fit f;
    if (n == 0) return f;
    if (n == 1) {
        f.b = (float)y[0];
        return f;
    }
    double mx = 0, my = 0;
    for (uint32_t i = 0; i < n; ++i) {
        mx += i;
        my += y[i];
    }
    mx /= n;
    my /= n;
    double sxx = 0, sxy = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const double dx = i - mx;
        sxx += dx * dx;
        sxy += dx * ((double)y[i] - my);
    }
    f.a = (float)(sxy / sxx);
    f.b = (float)(my - (double)f.a * mx);
    float left = 0, right = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const float d = ((float)y[i] - f.b) / f.a - (float)i;
        if (d > left) left = d;
        else if (d < right) right = d;
    }
    f.L = (uint32_t)left + 1u;
    f.R = (uint32_t)(0.0f - right) + 1u;
    return f;
}

struct FitLrc {
    float slope = 1.0f;
    int32_t icpt = 0;
    float range = 0.0f;
};

static FitLrc fit_lrc(const uint32_t *y, uint32_t n) {
    FitLrc f;
    if (n == 0) return f;
    if (n == 1) {
        f.icpt = (int32_t)y[0];
        return f;
    }
    double mx = 0, my = 0;
    for (uint32_t i = 0; i < n; ++i) {
        mx += i;
        my += y[i];
    }
    mx /= n;
    my /= n;
    double sxx = 0, sxy = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const double dx = i - mx;
        sxx += dx * dx;
        sxy += dx * ((double)y[i] - my);
    }
    const double s = sxy / sxx, c = my - s * mx;
    double left = 0, right = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const double d = ((double)y[i] - c) / s - i;
        if (d > left) left = d;
        else if (d < right) right = d;
    }
    f.slope = (float)s;
    f.icpt = (int32_t)c;
    f.range = (float)(left - right);
    return f;
}

void fit_lrc_host(const uint32_t *y, uint32_t n, float *slope, int32_t *icpt, float *range) {
    const FitLrc f = fit_lrc(y, n);
    *slope = f.slope;
    *icpt = f.icpt;
    *range = f.range;
}

// Float -> int32 truncation as the device evaluates it (cvt.rzi.s32.f32):
// out-of-range values saturate and NaN becomes 0. The reference's residuals
// were computed and are decoded on the GPU, so this is the format's semantics.
static inline int32_t f2i_sat(float v) {
    if (std::isnan(v)) return 0;
    if (v >= 2147483648.0f) return 2147483647;
    if (v <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)v;
}

// ---------------------------------------------------------------------------
// One list -> blocks + metadata.

void fixed_list_directory(ListDesc &d, const uint32_t *head, uint32_t ns, std::vector<uint32_t> &dir) {
    const int sh = (int)nbits(d.last_doc) - (int)nbits(ns);
    d.dir_shift = (uint32_t)std::max(sh, 0);
    d.ndir = (uint32_t)(((uint64_t)d.last_doc >> d.dir_shift) + 1);
    dir.assign((size_t)d.ndir + 1, 0);
    uint32_t s = 0;
    for (uint32_t b = 0; b <= d.ndir; ++b) {
        while (s < ns && ((uint64_t)head[s] >> d.dir_shift) < b) ++s;
        dir[b] = s;
    }
}

int32_t seg_pred_host(uint32_t idx, float a, float b) { return f2i_sat(std::fmaf((float)idx, a, b)); }

uint32_t lrc_pred_host(uint32_t idx, float slope, int32_t icpt) {
    return (uint32_t)f2i_sat((float)(int32_t)idx * slope) + (uint32_t)icpt;
}

int variable_list_tiles(const uint32_t *cnt, uint32_t ns, std::vector<uint64_t> &tiles) {
    // a segment larger than a tile is cut into 256-slices; consecutive small
    // segments are grouped while they fit in one tile
    uint32_t s = 0;
    while (s < ns) {
        if (cnt[s] >= kTileKeys) {
            if (cnt[s] > kTileMaxE0) return EXCL_E_FORMAT;
            for (uint32_t k = 0; k < cnt[s]; k += kTileKeys) tiles.push_back(tile_pack(s, k, 1));
            ++s;
            continue;
        }
        uint32_t keys = 0, g = 0;
        while (s + g < ns && g < kTileMaxSegs && cnt[s + g] < kTileKeys && keys + cnt[s + g] <= kTileKeys)
            keys += cnt[s + g++];
        tiles.push_back(tile_pack(s, 0, g));
        s += g;
    }
    return EXCL_OK;
}

SegReg fit_host(const uint32_t *y, uint32_t n) {
    const Fit f = fit_segment(y, n);
    return SegReg{f.a, f.b, f.L, f.R};
}

struct ListOut {
    ListDesc d{};
    std::vector<uint32_t> words, head, dir;
    std::vector<SegRec> rec;
    std::vector<SegReg> reg;
    std::vector<uint64_t> tiles;
    int status = EXCL_OK;
    std::string err;
};

static void fail(ListOut &o, int st, const std::string &m) {
    o.status = st;
    o.err = m;
}

// Fills segment boundaries (start, count) for the list's codec.
static void segment_list(const uint32_t *docs, uint32_t n, uint32_t codec, const excl_build_params &p,
                         ListOut &o, std::vector<uint32_t> &st, std::vector<uint32_t> &cnt,
                         std::vector<uint32_t> &bucket_first_seg) {
    if (!codec_is_hs(codec)) {
        const uint32_t B = p.block;
        const uint32_t ns = (n + B - 1) / B;
        for (uint32_t s = 0; s < ns; ++s) {
            st.push_back(s * B);
            cnt.push_back(std::min(B, n - s * B));
        }
        return;
    }
    // HS_SegLRC_Generator.cu:545-581: shift from the length (expected bucket
    // size), or the top kbits of a ubits-bit universe.
    const uint32_t maxb = nbits(docs[n - 1]);
    uint32_t shift;
    if (p.hs_kbits) {
        shift = p.hs_ubits > p.hs_kbits ? p.hs_ubits - p.hs_kbits : 0;
    } else if (n <= p.hs_bucket) {
        shift = maxb;
    } else {
        const uint32_t expect = (n + p.hs_bucket - 1) / p.hs_bucket;
        shift = maxb - nbits(expect);
    }
    const uint32_t nb = (uint32_t)(((uint64_t)docs[n - 1] >> shift) + 1);
    o.d.dir_shift = shift;
    o.d.ndir = nb;
    bucket_first_seg.assign(nb + 1, 0);
    const uint32_t B = (codec == EXCL_CODEC_HS_PARAPFD) ? p.block : 0xffffffffu;
    uint32_t i = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        bucket_first_seg[b] = (uint32_t)st.size();
        uint32_t j = i;
        while (j < n && ((uint64_t)docs[j] >> shift) == b) ++j;
        for (uint32_t k = i; k < j; k += std::min(B, j - k)) {
            st.push_back(k);
            cnt.push_back(std::min(B, j - k));
        }
        i = j;
    }
    bucket_first_seg[nb] = (uint32_t)st.size();
}

static void build_list(const uint32_t *docs, uint32_t n, uint32_t codec, const excl_build_params &p, ListOut &o) {
    if (n == 0) return fail(o, EXCL_E_INVALID, "empty posting list");
    for (uint32_t i = 1; i < n; ++i)
        if (docs[i] <= docs[i - 1]) return fail(o, EXCL_E_INVALID, "posting list not strictly increasing");
    ListDesc &d = o.d;
    d.n = n;
    d.codec = codec;
    d.first_doc = docs[0];
    d.last_doc = docs[n - 1];
    d.model = kNoModel;
    std::vector<uint32_t> st, cnt, bfirst;
    segment_list(docs, n, codec, p, o, st, cnt, bfirst);
    const uint32_t ns = (uint32_t)st.size();
    d.nseg = ns;
    d.log2_block = codec_is_hs(codec) ? 0u : (uint32_t)__builtin_ctz(p.block);

    // values to pack per element
    std::vector<uint32_t> val(n);
    o.rec.resize(ns);
    o.reg.assign(ns, SegReg{1.0f, 0.0f, 0, 0});
    if (codec_is_dgap(codec)) {
        // ParaPFD_Compression/main.cpp:163-186
        val[0] = docs[0];
        for (uint32_t j = 1; j < n; ++j) val[j] = docs[j] - docs[j - 1];
        for (uint32_t s = 0; s < ns; ++s) o.rec[s].aux = docs[st[s] + cnt[s] / 2];
    } else if (codec == EXCL_CODEC_LRC) {
        // LRC_Generator.cu:155-178 + LRC_Generator_kernel.cu:68-88
        FitLrc f = fit_lrc(docs, n);
        if (n > 1) {
            int32_t mn = 0;
            std::vector<int32_t> r(n);
            for (uint32_t i = 0; i < n; ++i) {
                const int32_t y = (int32_t)lrc_pred_host(i, f.slope, f.icpt);
                r[i] = (int32_t)(docs[i] - (uint32_t)y);
                if (i == 0 || r[i] < mn) mn = r[i];
            }
            for (uint32_t i = 0; i < n; ++i) {
                const int64_t v = (int64_t)r[i] - mn;
                if (v > 0x7fffffffLL) return fail(o, EXCL_E_FORMAT, "LRC residual spread exceeds 31 bits");
                val[i] = (uint32_t)v;
            }
            f.icpt = (int32_t)((uint32_t)f.icpt + (uint32_t)mn);
        } else {
            val[0] = 0;
        }
        std::memcpy(&d.reg[0], &f.slope, 4);
        std::memcpy(&d.reg[1], &f.icpt, 4);
        std::memcpy(&d.reg[2], &f.range, 4);
        d.reg[3] = 0;
    } else {
        // LRCSeg / SegLRC / HS_SegLRC: list fit (LRCSeg residual basis; SegLRC
        // list-level borders), per-segment fit for SegLRC/HS, per-segment base.
        const Fit lf = fit_segment(docs, n);
        std::memcpy(&d.reg[0], &lf.a, 4);
        std::memcpy(&d.reg[1], &lf.b, 4);
        d.reg[2] = lf.L;
        d.reg[3] = lf.R;
        std::vector<int32_t> r(n);
        for (uint32_t s = 0; s < ns; ++s) {
            const uint32_t s0 = st[s], c = cnt[s];
            Fit f = lf;
            if (codec != EXCL_CODEC_LRCSEG) {
                f = fit_segment(docs + s0, c);
                o.reg[s] = SegReg{f.a, f.b, f.L, f.R};
            }
            int32_t mn = 0;
            for (uint32_t k = 0; k < c; ++k) {
                const uint32_t idx = (codec == EXCL_CODEC_LRCSEG) ? s0 + k : k;
                const float pf = std::fmaf((float)idx, f.a, f.b);
                const int32_t y = f2i_sat(pf);
                const int32_t v = (int32_t)(docs[s0 + k] - (uint32_t)y);
                r[s0 + k] = v;
                if (k == 0 || v < mn) mn = v;
            }
            for (uint32_t k = 0; k < c; ++k) {
                const int64_t v = (int64_t)r[s0 + k] - mn;
                if (v > 0x7fffffffLL) return fail(o, EXCL_E_FORMAT, "residual spread exceeds 31 bits");
                val[s0 + k] = (uint32_t)v;
            }
            o.rec[s].aux = (uint32_t)mn;
        }
    }

    // ParaPFD blocks, one per segment.
    std::vector<uint32_t> tmp;
    o.head.resize(ns);
    for (uint32_t s = 0; s < ns; ++s) {
        const uint32_t c = cnt[s];
        tmp.assign((size_t)c * 3 + 8, 0u);
        int err = 0;
        const uint32_t w = codec_is_newpfd(codec) ? newpfd_encode_block(val.data() + st[s], c, p.frac, tmp.data(), &err)
                                                   : pfd_encode_block(val.data() + st[s], c, p.frac, tmp.data(), &err);
        if (err) return fail(o, err, "block not representable (b = 32, > 65535 exceptions, or a NewPFD high part > 28 bits)");
        o.rec[s].start = st[s];
        o.rec[s].off = (uint32_t)o.words.size();
        o.rec[s].count = c;
        o.head[s] = docs[st[s]];
        o.words.insert(o.words.end(), tmp.begin(), tmp.begin() + w);
    }

    // Directory: HS lists use their bucket table; fixed lists get a top-bits
    // directory with about one segment per bucket (cuda_hashSegment.cu:815-).
    if (codec_is_hs(codec)) {
        o.dir = bfirst;
    } else {
        fixed_list_directory(d, o.head.data(), ns, o.dir);
    }

    // Tiles (when this list is a query's shortest): one per fixed segment, or
    // one per 256-slice of a variable segment.
    if (d.log2_block) {
        d.ntiles = ns;
    } else {
        if (variable_list_tiles(cnt.data(), ns, o.tiles)) return fail(o, EXCL_E_FORMAT, "hash bucket larger than 2^24 postings");
        d.ntiles = (uint32_t)o.tiles.size();
    }
}

int build_index(const uint32_t *docs, const uint64_t *loff, uint32_t nlists, const excl_build_params &p,
                HostIndex &ix, std::string &err) {
    if (!docs || !loff || nlists == 0) {
        err = "null input or no lists";
        return EXCL_E_INVALID;
    }
    if (p.block < kMinBlock || p.block > kTileKeys || (p.block & (p.block - 1))) {
        err = "block must be a power of two in [32, 256]";
        return EXCL_E_INVALID;
    }
    for (uint32_t l = 0; l < nlists; ++l) {
        const uint32_t c = p.codecs ? p.codecs[l] : p.codec;
        if (c > EXCL_CODEC_NEWPFD) {
            err = "unknown codec";
            return EXCL_E_INVALID;
        }
        if (codec_is_hs(c) && !p.hs_kbits && p.hs_bucket == 0) {
            err = "HS codec needs hs_bucket or hs_kbits";
            return EXCL_E_INVALID;
        }
        if (loff[l + 1] < loff[l] || loff[l + 1] - loff[l] > 0xffffffffull) {
            err = "bad list offsets";
            return EXCL_E_INVALID;
        }
    }
    std::vector<ListOut> outs(nlists);
    unsigned nth = p.threads ? p.threads : std::max(1u, std::thread::hardware_concurrency());
    nth = std::min<unsigned>(nth, nlists);
    std::vector<std::thread> th;
    std::atomic_uint next{0};
    auto work = [&]() {
        for (;;) {
            const uint32_t l = next.fetch_add(1);
            if (l >= nlists) break;
            const uint32_t c = p.codecs ? p.codecs[l] : p.codec;
            build_list(docs + loff[l], (uint32_t)(loff[l + 1] - loff[l]), c, p, outs[l]);
        }
    };
    for (unsigned t = 0; t < nth; ++t) th.emplace_back(work);
    for (auto &t : th) t.join();

    ix.nlists = nlists;
    ix.lists.resize(nlists);
    uint64_t nw = 0, ns = 0, nd = 0, nt = 0;
    for (uint32_t l = 0; l < nlists; ++l) {
        if (outs[l].status) {
            err = "list " + std::to_string(l) + ": " + outs[l].err;
            return outs[l].status;
        }
        nw += outs[l].words.size();
        ns += outs[l].head.size();
        nd += outs[l].dir.size();
        nt += outs[l].tiles.size();
    }
    if (ns > 0xffffffffull || nd > 0xffffffffull || nt > 0xffffffffull) {
        err = "index too large for 32-bit segment indexing";
        return EXCL_E_CAPACITY;
    }
    ix.words.reserve(nw + kWordPad);
    ix.seg_head.reserve(ns);
    ix.seg_rec.reserve(ns);
    ix.seg_reg.reserve(ns);
    ix.dir.reserve(nd);
    ix.tilemap.reserve(nt);
    ix.postings = 0;
    for (uint32_t l = 0; l < nlists; ++l) {
        ListOut &o = outs[l];
        ListDesc d = o.d;
        d.word_base = ix.words.size();
        d.seg_base = (uint32_t)ix.seg_head.size();
        d.dir_base = (uint32_t)ix.dir.size();
        d.tile_base = (uint32_t)ix.tilemap.size();
        ix.lists[l] = d;
        ix.postings += d.n;
        ix.words.insert(ix.words.end(), o.words.begin(), o.words.end());
        ix.seg_head.insert(ix.seg_head.end(), o.head.begin(), o.head.end());
        ix.seg_rec.insert(ix.seg_rec.end(), o.rec.begin(), o.rec.end());
        ix.seg_reg.insert(ix.seg_reg.end(), o.reg.begin(), o.reg.end());
        ix.dir.insert(ix.dir.end(), o.dir.begin(), o.dir.end());
        ix.tilemap.insert(ix.tilemap.end(), o.tiles.begin(), o.tiles.end());
        ListOut().words.swap(o.words);
    }
    ix.words.resize(ix.words.size() + kWordPad, 0u);
    return EXCL_OK;
}

}  // namespace excl
