// Device helpers shared by the kernels: bit extraction from LSB-first packed
// ParaPFD sections, block headers, per-codec value reconstruction, the
// warp-cooperative block decode and the per-lane probe of one longer list.
#pragma once
#include <cuda_runtime.h>

#include "excl_internal.h"

namespace excl {

// Learned position model (two-stage): root MLP 1->32->32->1 on the normalized
// key routes to one of `nleaves` linear leaves; each leaf stores the exact
// rank error window of its keys, measured with this same inference code.
constexpr int kHidden = 32;
constexpr int kRootParams = kHidden + kHidden + kHidden * kHidden + kHidden + kHidden + 1;  // 1153
constexpr int kRootStride = 1156;

// The root is trained with non-negative weights, so its FP32 evaluation (and
// the leaf floor(out * L)) is non-decreasing in the key. Its routing is
// therefore a step function of the key and is stored exactly as the first key
// of every leaf (bnd) plus a coarse grid of the routing over the key range;
// the probe routes with two or three loads instead of evaluating the network.
struct alignas(16) ModelHdr {
    float kmin, kscale;    // x = (key - kmin) * kscale in [0, 1]
    uint32_t nleaves;      // leaves of this model
    uint32_t leaf_base;    // first leaf in the leaf array
    uint32_t n;            // postings of the list
    uint32_t max_window;   // leaves with a wider window fall back to the directory search
    uint32_t first;        // first docID of the list (grid origin)
    uint32_t grid_shift;   // grid cell = (key - first) >> grid_shift
    uint32_t grid_n;       // cells; the grid holds grid_n + 1 leaf ids
    uint32_t grid_base;    // first entry in the grid array
    uint32_t bnd_base;     // first entry in the boundary array (nleaves entries)
    uint32_t pad;
};

struct alignas(16) Leaf {
    float a, b;     // rank ~ a * x + b (x normalized key)
    int32_t elo;    // rank >= pred + elo for every key of the leaf (elo <= 0)
    int32_t ehi;    // rank <= pred + ehi
};

struct ModelView {
    const float *root = nullptr;      // kRootStride floats per model
    const ModelHdr *hdr = nullptr;
    const Leaf *leaves = nullptr;
    const uint16_t *grid = nullptr;   // routing at grid points
    const uint32_t *bnd = nullptr;    // bnd[l] = first key routed to a leaf >= l (0xffffffff: none)
};

struct DevIndexView {
    const ListDesc *lists;
    const uint32_t *words;
    const uint32_t *seg_head;
    const SegRec *seg_rec;
    const SegReg *seg_reg;
    const uint32_t *dir;
    const uint64_t *tilemap;
    const uint64_t *post_base;
    const uint32_t *seg_list;   // list of each segment
    const uint64_t *seg_gword;  // first word of each segment's block (nsegs + 1 entries)
    const ProbeRec *seg_probe;  // per-segment probe records
    ModelView models;
    uint32_t codec_mask;        // bit c set: some list of the index has codec c
};

// Tiles per fixed segment of a query's shortest list: 2^split, capped so a
// tile keeps at least kMinBlock (32) keys; variable (HS) lists are not cut.
__host__ __device__ inline uint32_t tile_split_of(uint32_t log2_block, uint32_t split) {
    return log2_block > 5u ? (split < log2_block - 5u ? split : log2_block - 5u) : 0u;
}

// Tiles of a shortest list of n postings and ntiles whole-segment tiles when
// fixed segments are cut: 2^s per segment, and only as many as the last
// segment's postings fill (so no tile is empty and a list of n postings never
// has more than n/32 + 1 tiles).
__host__ __device__ inline uint32_t split_tiles(uint32_t n, uint32_t ntiles, uint32_t log2_block, uint32_t split) {
    const uint32_t sp = tile_split_of(log2_block, split);
    if (!sp || ntiles == 0) return ntiles;
    const uint32_t last = n - ((ntiles - 1u) << log2_block), sub_log = log2_block - sp;
    return ((ntiles - 1u) << sp) + ((last + (1u << sub_log) - 1u) >> sub_log);
}

// Codec families a kernel instance is compiled for; an index whose lists all
// belong to one family launches the narrower instance (fewer registers).
enum : int { kKindAny = 0, kKindResid = 1, kKindDgap = 2 };
__host__ __device__ inline int codec_kind(uint32_t mask) {
    const uint32_t resid = (1u << EXCL_CODEC_LRC) | (1u << EXCL_CODEC_LRCSEG) | (1u << EXCL_CODEC_SEGLRC) |
                           (1u << EXCL_CODEC_HS_SEGLRC);
    const uint32_t dgap = (1u << EXCL_CODEC_PARAPFD) | (1u << EXCL_CODEC_HS_PARAPFD);
    if (mask && !(mask & ~resid)) return kKindResid;
    if (mask && !(mask & ~dgap)) return kKindDgap;
    return kKindAny;
}

enum : uint32_t {
    kErrTerms = 1u,      // a query has more than kMaxTerms terms
    kErrScanSpin = 2u,   // a look-back wait gave up
    kErrTermId = 4u,     // a term id is out of range
    kErrCapacity = 8u,   // results or tiles exceed a buffer
    kErrModel = 16u,     // learned model inconsistency
};

__device__ __forceinline__ uint32_t ldg(const uint32_t *p) { return __ldg(p); }

// `bits` (0..31) bits starting at bit `bitpos` of the packed array `w`.
// Reads two words; the index keeps kWordPad zero words after the last block.
__device__ __forceinline__ uint32_t get_bits(const uint32_t *w, uint32_t bitpos, uint32_t bits) {
    const uint32_t i = bitpos >> 5;
    const uint32_t lo = ldg(w + i), hi = ldg(w + i + 1);
    return __funnelshift_r(lo, hi, bitpos & 31u) & ((1u << bits) - 1u);
}

struct BlkHdr {
    uint32_t lb, eb, hb, en;
};

// ParaPFor.cpp:102-106 descriptor fields.
__device__ __forceinline__ BlkHdr blk_hdr(uint32_t d) {
    BlkHdr h;
    h.lb = (d >> 26) & 31u;
    h.eb = (d >> 21) & 31u;
    h.hb = (d >> 16) & 31u;
    h.en = d & 0xffffu;
    return h;
}

__device__ __forceinline__ uint32_t words_for(uint32_t n, uint32_t bits) { return (n * bits + 31u) >> 5; }

// Predicted values of the regression codecs, with the reference's arithmetic:
// LRC (LRC_Decompression_kernel.cu:254): int((float)i * slope) + icpt;
// LRCSeg/SegLRC/HS (SegLRC_Decompression_kernel.cu:252): (int)(i * a + b) as
// one fused multiply-add.
__device__ __forceinline__ uint32_t pred_lrc(uint32_t i, float slope, int32_t icpt) {
    return (uint32_t)__float2int_rz(__fmul_rn(__int2float_rn((int)i), slope)) + (uint32_t)icpt;
}
__device__ __forceinline__ uint32_t pred_fma(uint32_t i, float a, float b) {
    return (uint32_t)__float2int_rz(__fmaf_rn(__uint2float_rn(i), a, b));
}

// Per-segment reconstruction parameters of a residual-coded segment:
// value(t) = low(t) + pred(idx0 + t) + base.
struct ResidParams {
    float a, b;
    uint32_t idx0;   // index fed to the predictor for t = 0
    uint32_t base;   // added after the prediction (LRC: the intercept)
    bool lrc;
};

__device__ __forceinline__ ResidParams resid_params(const ListDesc &L, const SegRec &rec, const SegReg &reg) {
    ResidParams p;
    if (L.codec == EXCL_CODEC_LRC) {
        p.a = __uint_as_float(L.reg[0]);
        p.b = 0.0f;
        p.idx0 = rec.start;
        p.base = L.reg[1];
        p.lrc = true;
    } else if (L.codec == EXCL_CODEC_LRCSEG) {
        p.a = __uint_as_float(L.reg[0]);
        p.b = __uint_as_float(L.reg[1]);
        p.idx0 = rec.start;
        p.base = rec.aux;
        p.lrc = false;
    } else {
        p.a = reg.a;
        p.b = reg.b;
        p.idx0 = 0;
        p.base = rec.aux;
        p.lrc = false;
    }
    return p;
}

__device__ __forceinline__ uint32_t resid_value(const ResidParams &p, uint32_t t, uint32_t low) {
    const uint32_t i = p.idx0 + t;
    return low + (p.lrc ? pred_lrc(i, p.a, (int32_t)p.base) : pred_fma(i, p.a, p.b) + p.base);
}

// Low bits of element t of a block plus its exception high bits, by binary
// search over the sorted exception positions (random access).
__device__ __forceinline__ uint32_t block_value_ra(const uint32_t *blk, const BlkHdr &h, uint32_t count, uint32_t t) {
    uint32_t v = get_bits(blk + 1, t * h.lb, h.lb);
    if (h.en) {
        const uint32_t *pb = blk + 1 + words_for(count, h.lb);
        uint32_t lo = 0, hi = h.en;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (get_bits(pb, mid * h.eb, h.eb) < t) lo = mid + 1;
            else hi = mid;
        }
        if (lo < h.en && get_bits(pb, lo * h.eb, h.eb) == t) {
            const uint32_t *hp = pb + words_for(h.en, h.eb);
            v |= get_bits(hp, lo * h.hb, h.hb) << h.lb;
        }
    }
    return v;
}

// ---------------------------------------------------------------------------
// NewPFD exceptions: one Simple-16 stream (NewPFor.cpp:91-106) holding the
// exception positions (first absolute, then gaps minus one) and then their
// high parts. Two cursors walk it in step: one over the positions, one
// started past them over the high parts.

// Simple-16 word layouts (the published 16 cases; also the reference's
// Simple16.h): up to three runs of (count, width), low bits first.
static __constant__ uint8_t kS16Dev[16][6] = {
    {28, 1, 0, 0, 0, 0}, {7, 2, 14, 1, 0, 0}, {7, 1, 7, 2, 7, 1}, {14, 1, 7, 2, 0, 0},
    {14, 2, 0, 0, 0, 0}, {1, 4, 8, 3, 0, 0},  {1, 3, 4, 4, 3, 3}, {7, 4, 0, 0, 0, 0},
    {4, 5, 2, 4, 0, 0},  {2, 4, 4, 5, 0, 0},  {3, 6, 2, 5, 0, 0}, {2, 5, 3, 6, 0, 0},
    {4, 7, 0, 0, 0, 0},  {1, 10, 2, 9, 0, 0}, {2, 14, 0, 0, 0, 0}, {1, 28, 0, 0, 0, 0}};

struct S16Cursor {
    const uint32_t *p;  // current word (global or shared memory)
    uint32_t word, j, sh, left, run, width;  // value j of the word; `left` values remain in the current run
};

__device__ __forceinline__ void s16_load(S16Cursor &c) {
    c.word = *c.p;
    const uint32_t k = c.word >> 28;
    c.j = 0;
    c.sh = 0;
    c.run = 0;
    c.left = kS16Dev[k][0];
    c.width = kS16Dev[k][1];
}

__device__ __forceinline__ void s16_start(S16Cursor &c, const uint32_t *p) {
    c.p = p;
    s16_load(c);
}

__device__ __forceinline__ uint32_t s16_next(S16Cursor &c) {
    while (c.left == 0) {  // next run of the word, or the next word
        const uint32_t k = c.word >> 28;
        if (++c.run < 3 && kS16Dev[k][2 * c.run]) {
            c.left = kS16Dev[k][2 * c.run];
            c.width = kS16Dev[k][2 * c.run + 1];
        } else {
            ++c.p;
            s16_load(c);
        }
    }
    const uint32_t v = (c.word >> c.sh) & ((1u << c.width) - 1u);  // widths are <= 28
    c.sh += c.width;
    --c.left;
    return v;
}

// Values in a Simple-16 word, and value j of it (its runs of (count, width),
// low bits first).
__device__ __forceinline__ uint32_t s16_count(uint32_t word) {
    const uint32_t k = word >> 28;
    return (uint32_t)kS16Dev[k][0] + kS16Dev[k][2] + kS16Dev[k][4];
}
__device__ __forceinline__ uint32_t s16_value(uint32_t word, uint32_t j) {
    const uint32_t k = word >> 28;
    const uint32_t c0 = kS16Dev[k][0], w0 = kS16Dev[k][1], c1 = kS16Dev[k][2], w1 = kS16Dev[k][3],
                   w2 = kS16Dev[k][5];
    uint32_t off, wd;
    if (j < c0) {
        off = j * w0;
        wd = w0;
    } else if (j < c0 + c1) {
        off = c0 * w0 + (j - c0) * w1;
        wd = w1;
    } else {
        off = c0 * w0 + c1 * w1 + (j - c0 - c1) * w2;
        wd = w2;
    }
    return (word >> off) & ((1u << wd) - 1u);  // widths are <= 28
}

// Group-parallel patch of a NewPFD block's exceptions: at(pos - e0) += high
// << b for every exception at a position in [e0, e0 + kc). The block's
// Simple-16 stream (NewPFor.cpp:91-106) holds the en position codes (the
// first absolute, then gaps minus one) and then the en high parts; `nw` words
// of it may be read. The warp works in groups of G = 2^lg lanes (sub = lane
// within the group, one block per group); every lane of the warp calls this,
// and a group with en = 0 only keeps step. Per round of G exceptions: the
// group scans the value counts of G stream words at a time (each lane one
// word's selector), so every word's first value index is known, and each lane
// finds the words holding its exception's position code and high part with a
// search over the group's word starts (shuffles); a group scan of the codes
// then gives the positions. The reference decodes this stream with one thread
// of a block (NewPFD_Decompression_kernel.cu:432-440).
template <class At>
__device__ __forceinline__ void newpfd_patch_group(const uint32_t *s16, uint32_t nw, uint32_t en, uint32_t b,
                                                   uint32_t e0, uint32_t kc, uint32_t lg, uint32_t sub, At at) {
    const uint32_t G = 1u << lg, full = 0xffffffffu;
    const uint32_t nwv = min(nw, 2u * en);  // a stream of 2 en values has at most 2 en words
    // trip counts the whole warp shares (shuffles need every lane)
    const uint32_t xrounds = __reduce_max_sync(full, (en + G - 1u) >> lg);
    const uint32_t wrounds = __reduce_max_sync(full, (nwv + G - 1u) >> lg);
    uint32_t pcarry = 0;  // position of the previous round's last exception
    for (uint32_t xr = 0; xr < xrounds; ++xr) {
        const uint32_t x = (xr << lg) + sub;
        const bool live = x < en;
        uint32_t code = 0, high = 0, vstart = 0;
        for (uint32_t wr = 0; wr < wrounds; ++wr) {
            const uint32_t wi = (wr << lg) + sub;
            const uint32_t word = wi < nwv ? s16[wi] : 0u;
            const uint32_t cnt = wi < nwv ? s16_count(word) : 0u;
            uint32_t inc = cnt;
            for (uint32_t o = 1; o < G; o <<= 1) {
                const uint32_t t = __shfl_up_sync(full, inc, o, G);
                if (sub >= o) inc += t;
            }
            const uint32_t st = vstart + inc - cnt;  // value index of this lane's word
            const uint32_t total = __shfl_sync(full, inc, G - 1u, G);
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const uint32_t k = r ? en + x : x;
                // the last lane of the group whose word starts at or before k
                uint32_t lo = 0;
                for (uint32_t hb = G >> 1; hb; hb >>= 1) {
                    const uint32_t sv = __shfl_sync(full, st, lo + hb, G);
                    if (sv <= k) lo += hb;
                }
                const uint32_t wv = __shfl_sync(full, word, lo, G), sv = __shfl_sync(full, st, lo, G);
                if (live && k >= vstart && k < vstart + total) {
                    const uint32_t v = s16_value(wv, k - sv);
                    if (r) high = v;
                    else code = v;
                }
            }
            vstart += total;
        }
        // positions: p(0) = code(0), p(x) = p(x - 1) + code(x) + 1
        const uint32_t d = live ? code + (x ? 1u : 0u) : 0u;
        uint32_t inc = d;
        for (uint32_t o = 1; o < G; o <<= 1) {
            const uint32_t t = __shfl_up_sync(full, inc, o, G);
            if (sub >= o) inc += t;
        }
        const uint32_t p = pcarry + inc;
        if (live && p >= e0 && p < e0 + kc) at(p - e0) += high << b;
        pcarry = __shfl_sync(full, p, G - 1u, G);
    }
}

// Warp-cooperative decode of elements [e0, e0 + kc) (kc <= 256) of one
// segment into buf[0 .. kc). Lane l owns elements l*vpl .. l*vpl+vpl-1 so its
// bits are contiguous; exceptions are patched through `buf`; d-gap codecs
// replace element 0 by the segment head and take a warp inclusive scan
// (ParaPFD_Decompression_kernel.cu:205-263), residual codecs add the
// regression prediction and base (SegLRC_Decompression_kernel.cu:249-252).
template <int KIND = kKindAny>
__device__ __forceinline__ void warp_decode(const DevIndexView &ix, const ListDesc &L, uint32_t sg, uint32_t e0,
                                            uint32_t kc, uint32_t *buf, uint32_t lane) {
    const bool dgap = KIND == kKindDgap || (KIND == kKindAny && codec_is_dgap(L.codec));
    const bool newpfd = KIND == kKindAny && codec_is_newpfd(L.codec);
    // the segment's 64-byte probe record: head, block offset, aux, count,
    // descriptor, regression and list position, all in one round trip (no
    // dependent load of the block's descriptor word before its bits)
    const uint4 *prv = reinterpret_cast<const uint4 *>(ix.seg_probe + sg);
    const uint4 p0 = __ldg(prv), p1 = __ldg(prv + 1), p2 = __ldg(prv + 2);
    SegRec rec;
    rec.off = p0.y;
    rec.aux = p0.z;
    rec.count = p0.w;
    rec.start = p2.x;
    const uint32_t *blk = ix.words + L.word_base + rec.off;
    const BlkHdr h = blk_hdr(p1.x);
    const uint32_t vpl = (kc + 31u) >> 5;
    const uint32_t el = lane * vpl;
    uint32_t v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t e = el + j;
        v[j] = (j < (int)vpl && e < kc) ? get_bits(blk + 1, (e0 + e) * h.lb, h.lb) : 0u;
    }
    if (h.en) {
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j < (int)vpl && el + j < kc) buf[el + j] = v[j];
        __syncwarp();
        const uint32_t *pb = blk + 1 + words_for(rec.count, h.lb);
        if (newpfd) {
            // the stream ends with the block: its words from the block's extent
            const uint32_t bw = (uint32_t)(__ldg(ix.seg_gword + sg + 1) - __ldg(ix.seg_gword + sg));
            const uint32_t nw = bw - 1u - words_for(rec.count, h.lb);
            newpfd_patch_group(pb, nw, h.en, h.lb, e0, kc, 5u, lane,
                               [buf](uint32_t i) -> uint32_t & { return buf[i]; });
        } else {
            const uint32_t *hp = pb + words_for(h.en, h.eb);
            for (uint32_t x = lane; x < h.en; x += 32) {
                const uint32_t p = get_bits(pb, x * h.eb, h.eb);
                if (p >= e0 && p < e0 + kc) buf[p - e0] |= get_bits(hp, x * h.hb, h.hb) << h.lb;
            }
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j < (int)vpl && el + j < kc) v[j] = buf[el + j];
        __syncwarp();
    }
    if (dgap) {
        if (lane == 0 && e0 == 0) v[0] = p0.x;
        uint32_t run = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            run += v[j];
            v[j] = run;
        }
        uint32_t incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        const uint32_t excl = incl - run;
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] += excl;
    } else {
        SegReg reg;
        reg.a = __uint_as_float(p1.y);
        reg.b = __uint_as_float(p1.z);
        const ResidParams rp = resid_params(L, rec, reg);
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = resid_value(rp, e0 + el + j, v[j]);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if (j < (int)vpl && el + j < kc) buf[el + j] = v[j];
    __syncwarp();
}

// Last segment in [lo, hi) whose head <= key, or -1.
__device__ __forceinline__ int last_head_le(const uint32_t *head, uint32_t lo, uint32_t hi, uint32_t key) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (ldg(head + mid) <= key) lo = mid + 1;
        else hi = mid;
    }
    return (int)lo - 1;
}

// Last segment in [lo, hi) of a list's probe records whose head <= key, or lo - 1.
// Ranges of up to four records (the directory's usual one or two) load every
// head at once, one round trip instead of a chain of dependent loads.
__device__ __forceinline__ int last_head_le_rec(const ProbeRec *pr, uint32_t lo, uint32_t hi, uint32_t key) {
    if (hi - lo <= 4u && lo < hi) {
        uint32_t h[4];
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) h[j] = lo + j < hi ? __ldg(&pr[lo + j].head) : 0xffffffffu;
        int s = (int)lo - 1;
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j)
            if (lo + j < hi && h[j] <= key) s = (int)(lo + j);
        return s;
    }
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&pr[mid].head) <= key) lo = mid + 1;
        else hi = mid;
    }
    return (int)lo - 1;
}

// Serial search of `key` (head <= key) in a d-gap segment, starting at the
// segment head or at its median (ParaPFD_Intersection_kernel.cu:383-447:
// median halves the walk; exceptions tracked with a cursor).
__device__ __forceinline__ bool dgap_find(const uint32_t *blk, const BlkHdr h, uint32_t count, uint32_t head,
                                          uint32_t median, uint32_t key) {
    if (key == head || key == median) return true;
    uint32_t from, end, v;
    if (key > median) {
        from = count >> 1;
        end = count;
        v = median;
    } else {
        from = 0;
        end = count >> 1;
        v = head;
    }
    const uint32_t *lows = blk + 1;
    const uint32_t *pb = lows + words_for(count, h.lb);
    const uint32_t *hp = pb + words_for(h.en, h.eb);
    uint32_t x = 0, xp = 0xffffffffu;
    if (h.en) {
        uint32_t lo = 0, hi = h.en;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (get_bits(pb, mid * h.eb, h.eb) <= from) lo = mid + 1;
            else hi = mid;
        }
        x = lo;
        xp = x < h.en ? get_bits(pb, x * h.eb, h.eb) : 0xffffffffu;
    }
    // stream the low bits with a 64-bit window
    uint32_t bit = (from + 1) * h.lb;
    uint32_t wi = bit >> 5;
    uint64_t win = ((uint64_t)ldg(lows + wi + 1) << 32) | ldg(lows + wi);
    uint32_t sh = bit & 31u;
    const uint32_t mask = (1u << h.lb) - 1u;
    for (uint32_t i = from + 1; i < end; ++i) {
        uint32_t g = (uint32_t)(win >> sh) & mask;
        sh += h.lb;
        if (sh >= 32) {
            sh -= 32;
            ++wi;
            win = (win >> 32) | ((uint64_t)ldg(lows + wi + 1) << 32);
        }
        if (i == xp) {
            g |= get_bits(hp, x * h.hb, h.hb) << h.lb;
            ++x;
            xp = x < h.en ? get_bits(pb, x * h.eb, h.eb) : 0xffffffffu;
        }
        v += g;
        if (v >= key) return v == key;
    }
    return false;
}

// dgap_find for a NewPFD block: the same walk, exceptions read from the
// block's Simple-16 stream with two cursors.
__device__ __forceinline__ bool dgap_find_newpfd(const uint32_t *blk, const BlkHdr h, uint32_t count, uint32_t head,
                                                 uint32_t median, uint32_t key) {
    if (key == head || key == median) return true;
    uint32_t from, end, v;
    if (key > median) {
        from = count >> 1;
        end = count;
        v = median;
    } else {
        from = 0;
        end = count >> 1;
        v = head;
    }
    const uint32_t *lows = blk + 1;
    S16Cursor pc, hc;
    uint32_t x = 0, p = 0, xp = 0xffffffffu, xh = 0;
    if (h.en) {
        const uint32_t *s16 = lows + words_for(count, h.lb);
        s16_start(pc, s16);
        s16_start(hc, s16);
        for (uint32_t i = 0; i < h.en; ++i) s16_next(hc);
        // the first exception after `from`
        do {
            p = x ? p + s16_next(pc) + 1u : s16_next(pc);
            xh = s16_next(hc);
            ++x;
        } while (p <= from && x < h.en);
        xp = p > from ? p : 0xffffffffu;
    }
    uint32_t bit = (from + 1) * h.lb;
    uint32_t wi = bit >> 5;
    uint64_t win = ((uint64_t)ldg(lows + wi + 1) << 32) | ldg(lows + wi);
    uint32_t sh = bit & 31u;
    const uint32_t mask = (1u << h.lb) - 1u;
    for (uint32_t i = from + 1; i < end; ++i) {
        uint32_t g = (uint32_t)(win >> sh) & mask;
        sh += h.lb;
        if (sh >= 32) {
            sh -= 32;
            ++wi;
            win = (win >> 32) | ((uint64_t)ldg(lows + wi + 1) << 32);
        }
        if (i == xp) {
            g += xh << h.lb;
            if (x < h.en) {
                p += s16_next(pc) + 1u;
                xh = s16_next(hc);
                ++x;
                xp = p;
            } else {
                xp = 0xffffffffu;
            }
        }
        v += g;
        if (v >= key) return v == key;
    }
    return false;
}

// Binary search for `key` over elements [t0, t1] of a residual-coded segment.
__device__ __forceinline__ bool resid_find(const uint32_t *blk, const BlkHdr &h, const ResidParams &rp, uint32_t count,
                                           int t0, int t1, uint32_t key) {
    while (t0 <= t1) {
        const int mid = (t0 + t1) >> 1;
        const uint32_t v = resid_value(rp, (uint32_t)mid, block_value_ra(blk, h, count, (uint32_t)mid));
        if (v == key) return true;
        if (v < key) t0 = mid + 1;
        else t1 = mid - 1;
    }
    return false;
}

// Learned model inference (root MLP + leaf) -> predicted rank and the leaf.
// Every operation is an explicit round-to-nearest intrinsic so that the error
// bounds measured at build time hold bit for bit at query time.
__device__ __forceinline__ float model_root(const float *W, float x) {
    const float *w1 = W, *b1 = W + kHidden, *w2 = W + 2 * kHidden, *b2 = w2 + kHidden * kHidden,
                *w3 = b2 + kHidden, *b3 = w3 + kHidden;
    float h1[kHidden];
#pragma unroll
    for (int i = 0; i < kHidden; ++i) h1[i] = fmaxf(__fmaf_rn(w1[i], x, b1[i]), 0.0f);
    float out = b3[0];
#pragma unroll 4
    for (int o = 0; o < kHidden; ++o) {
        float acc = b2[o];
        const float *row = w2 + o * kHidden;
#pragma unroll
        for (int i = 0; i < kHidden; ++i) acc = __fmaf_rn(row[i], h1[i], acc);
        out = __fmaf_rn(w3[o], fmaxf(acc, 0.0f), out);
    }
    return out;
}

__device__ __forceinline__ uint32_t model_leaf_of(float root_out, uint32_t nleaves) {
    const float f = __fmul_rn(root_out, (float)nleaves);
    int li = __float2int_rd(f);
    li = li < 0 ? 0 : (li >= (int)nleaves ? (int)nleaves - 1 : li);
    return (uint32_t)li;
}

__device__ __forceinline__ float model_norm(const ModelHdr &m, uint32_t key) {
    return __fmul_rn(__fsub_rn(__uint2float_rn(key), m.kmin), m.kscale);
}

// Leaf of `key` (first <= key <= last) from the stored routing: the grid cell
// bounds the leaf to [grid[j], grid[j+1]]; the boundaries resolve it exactly.
__device__ __forceinline__ uint32_t model_route(const uint16_t *grid, const uint32_t *bnd, const ModelHdr &m,
                                                uint32_t key) {
    const uint32_t j = (key - m.first) >> m.grid_shift;
    uint32_t lo = grid[m.grid_base + j];
    uint32_t hi = grid[m.grid_base + j + 1];
    const uint32_t *b = bnd + m.bnd_base;
    if (hi - lo <= 8) {
        while (lo < hi && __ldg(b + lo + 1) <= key) ++lo;
        return lo;
    }
    // many leaves inside one cell: last l in [lo, hi] with b[l] <= key
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(b + mid) <= key) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int model_pred_rank(const Leaf &lf, float x) {
    const float r = __fmaf_rn(lf.a, x, lf.b);
    // clamp before the conversion so the result is defined
    const float rc = fminf(fmaxf(r, -1.0e9f), 1.0e9f);
    return __float2int_rd(rc);
}

}  // namespace excl
