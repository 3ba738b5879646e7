// The reference's on-disk index and query files, read and written as they are,
// so an index produced by its encoders runs here unchanged and an index built
// here can be handed to its binaries.
//
// File sets (`<dir>/<name><suffix>`; the reference keeps the regression files
// in a second directory, here they sit beside the others):
//
//   ParaPFD / NewPFD (ParaPFD_Compression/main.cpp:81-232, SegmentSize 256)
//     .ind1        per list {u32 length; u64 byte offset into .ind2}, 16 bytes
//                  with the x86-64 padding after length (main.cpp:32-35)
//     .ind2        the lists' blocks, list after list
//     .segNum      u32 per list: index of its first segment
//     .segHead     u32 per segment: its first docID
//     .segMedian   u32 per segment: docID at count / 2
//     .segOffset   u32 per segment: word offset of its block within the list
//   SegLRC (SegLRC_Compression/main.cpp:80-207, SegLRC_Generator.cu:94-436)
//     .ind1 .ind2 .segNum .segHead .segOffset as above (blocks of residuals)
//     .ind2_distance_base     i32 per segment: the residuals' minimum
//     .regression_info        per segment {float a; float b; u32 L; u32 R}
//     .regression_info_list   per list, same record (list-level fit)
//   LRC (LRC_Compression/main.cpp:94-215, LRC_Generator.cu:96-191)
//     .ind1 .ind2 .segNum .segHead .segOffset as above
//     .regression_info        per list {float slope; i32 intercept; float range}
//   LRCSeg (LRCSeg_Compression/main.cpp:78-200, LRCSeg_Generator.cu:98-215)
//     .ind1 .ind2 .segNum .segHead .segOffset .ind2_distance_base as SegLRC
//     .regression_info        per list {float a; float b; u32 L; u32 R}
//   HS_SegLRC (HS_SegLRC_Generator.cu:180-594, HS_SegLRC_Compression/main.cpp:78-190)
//     .ind1 .ind2 as above; one block per non-empty hash bucket
//     .HashSeg_offset         u32 per list: its record's word offset in .HashSeg_info
//     .HashSeg_info           per list {shift; buckets B; element offset of each
//                             bucket, B + 1 of them (the last is the length)}
//     .segNum                 u32 per list: index of its first bucket
//     .segOffset              u32 per bucket: word offset of its block within the
//                             list (an empty bucket: where the next block starts)
//     .ind2_distance_base     i32 per bucket: the residuals' minimum
//     .regression_info        per bucket {float a; float b; u32 L; u32 R}
//   Queries (ParaPFD_Intersection.cu:139-142)
//     .query       per query u32 term count, then that many u32 term ids
//
// The layout of these arrays is the layout of this library's index (lists and
// segments in the same order, the same block bytes, word offsets within the
// list), so loading copies them and derives the rest (segment counts and
// starts, last docIDs, directories, tile maps).
//
// Empty hash buckets. The reference's HS generator and decoder find an
// element's bucket by a lower-bound search over the bucket offsets
// (HS_SegLRC_Generator_kernel.cu:73-85, HS_SegLRC_Decompression_kernel.cu:
// 244-257), which hands the first element of a bucket that follows empty
// buckets to the first of those empty buckets: that element's residual and its
// decode use the empty bucket's fit, and it comes back wrong (the results the
// reference's HS path loses). This writer computes every residual against the
// element's own bucket, so a list without empty buckets is written byte for
// byte as the reference writes it and one with empty buckets decodes exactly
// here. An empty bucket's record is written as the generator leaves it: fit
// {1, 0, 0, 0} and, as base, the next element's docID. The loader rejects a
// set whose buckets do not decode to their own docID ranges.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "excl_internal.h"

using namespace excl;

namespace {

constexpr uint32_t kRefSegment = 256;  // SegmentSize of the reference encoders (and kExceptedBucketSize)

struct Ind1 {
    uint32_t length;
    uint32_t pad;
    uint64_t offset;
};
static_assert(sizeof(Ind1) == 16, "the reference's at_term_ind1_t is 16 bytes");

// LRC's per-list record (LRC_Generator_kernel.cu:37-41).
struct LrcReg {
    float slope;
    int32_t icpt;
    float range;
};
static_assert(sizeof(LrcReg) == 12, "the reference's LRC regression_info_t is 12 bytes");

std::string path_of(const char *dir, const char *name, const char *suffix) {
    std::string p = dir ? dir : ".";
    if (!p.empty() && p.back() != '/') p += '/';
    return p + name + suffix;
}

bool write_file(const std::string &p, const void *data, size_t bytes) {
    FILE *f = std::fopen(p.c_str(), "wb");
    if (!f) return false;
    const bool ok = bytes == 0 || std::fwrite(data, 1, bytes, f) == bytes;
    return std::fclose(f) == 0 && ok;
}

template <class T>
bool read_file(const std::string &p, std::vector<T> &out) {
    FILE *f = std::fopen(p.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0 || sz % (long)sizeof(T)) {
        std::fclose(f);
        return false;
    }
    out.resize((size_t)sz / sizeof(T));
    const bool ok = sz == 0 || std::fread(out.data(), 1, (size_t)sz, f) == (size_t)sz;
    std::fclose(f);
    return ok;
}

bool fixed_codec(uint32_t c) {
    return c == EXCL_CODEC_PARAPFD || c == EXCL_CODEC_SEGLRC || c == EXCL_CODEC_NEWPFD || c == EXCL_CODEC_LRC ||
           c == EXCL_CODEC_LRCSEG;
}

bool reference_codec(uint32_t c) { return fixed_codec(c) || c == EXCL_CODEC_HS_SEGLRC; }

uint32_t nbits32(uint32_t v) { return v ? 32u - (uint32_t)__builtin_clz(v) : 0u; }

// The reference's bucket shift for a list (HS_SegLRC_Generator.cu:545-557).
uint32_t ref_hs_shift(uint32_t n, uint32_t last) {
    const uint32_t maxb = nbits32(last);
    if (n <= kRefSegment) return maxb;
    return maxb - nbits32((n + kRefSegment - 1) / kRefSegment);
}

std::vector<Ind1> ind1_of(const excl_index *ix) {
    std::vector<Ind1> ind1(ix->nlists);
    for (uint32_t l = 0; l < ix->nlists; ++l) ind1[l] = Ind1{ix->lists[l].n, 0u, ix->lists[l].word_base * 4};
    return ind1;
}

int save_hs(const excl_index *ix, const char *dir, const char *name) {
    std::vector<uint32_t> hinfo, hoff(ix->nlists), bnum(ix->nlists), boff, base;
    std::vector<SegReg> reg;
    for (uint32_t l = 0; l < ix->nlists; ++l) {
        const ListDesc &d = ix->lists[l];
        // the reference's bucketing: shift from the length, one block per bucket
        if (d.dir_shift != ref_hs_shift(d.n, d.last_doc) || d.ndir != (d.last_doc >> d.dir_shift) + 1u)
            return EXCL_E_FORMAT;
        hoff[l] = (uint32_t)hinfo.size();
        bnum[l] = (uint32_t)boff.size();
        hinfo.push_back(d.dir_shift);
        hinfo.push_back(d.ndir);
        const uint32_t *bd = ix->dir.data() + d.dir_base;
        for (uint32_t b = 0; b < d.ndir; ++b) {
            if (bd[b + 1] - bd[b] > 1u) return EXCL_E_FORMAT;  // a bucket cut into several blocks
            const size_t g = (size_t)d.seg_base + bd[b];  // this bucket's block, or the next one
            hinfo.push_back(ix->seg_rec[g].start);
            boff.push_back(ix->seg_rec[g].off);
            if (bd[b + 1] > bd[b]) {
                base.push_back(ix->seg_rec[g].aux);
                reg.push_back(ix->seg_reg[g]);
            } else {
                base.push_back(ix->seg_head[g]);
                reg.push_back(SegReg{1.0f, 0.0f, 0u, 0u});
            }
        }
        hinfo.push_back(d.n);
    }
    const std::vector<Ind1> ind1 = ind1_of(ix);
    const uint64_t nwords = ix->words.size() - kWordPad;
    const bool ok = write_file(path_of(dir, name, ".ind1"), ind1.data(), ind1.size() * sizeof(Ind1)) &&
                    write_file(path_of(dir, name, ".ind2"), ix->words.data(), nwords * 4) &&
                    write_file(path_of(dir, name, ".HashSeg_offset"), hoff.data(), hoff.size() * 4) &&
                    write_file(path_of(dir, name, ".HashSeg_info"), hinfo.data(), hinfo.size() * 4) &&
                    write_file(path_of(dir, name, ".segNum"), bnum.data(), bnum.size() * 4) &&
                    write_file(path_of(dir, name, ".segOffset"), boff.data(), boff.size() * 4) &&
                    write_file(path_of(dir, name, ".ind2_distance_base"), base.data(), base.size() * 4) &&
                    write_file(path_of(dir, name, ".regression_info"), reg.data(), reg.size() * sizeof(SegReg));
    return ok ? EXCL_OK : EXCL_E_INVALID;
}

// Words of the block at `blk` (count values), or ~0 if it does not fit in `avail`.
uint64_t block_words(uint32_t codec, const uint32_t *blk, uint32_t count, uint64_t avail) {
    if (avail == 0) return ~0ull;
    const uint64_t w = codec == EXCL_CODEC_NEWPFD ? newpfd_block_words(blk, count, avail) : pfd_block_words(blk, count);
    return w <= avail ? w : ~0ull;
}

// The words array of a loaded set, padded as the index expects; empty on a bad size.
void take_words(excl_index *ix, std::vector<uint32_t> &ind2) {
    ix->words = std::move(ind2);
    ix->words.resize(ix->words.size() + kWordPad, 0u);
}

int load_hs(const char *dir, const char *name, excl_index **out) {
    std::vector<Ind1> ind1;
    std::vector<uint32_t> ind2, hoff, hinfo, bnum, boff, base;
    std::vector<SegReg> reg;
    if (!read_file(path_of(dir, name, ".ind1"), ind1) || !read_file(path_of(dir, name, ".ind2"), ind2) ||
        !read_file(path_of(dir, name, ".HashSeg_offset"), hoff) ||
        !read_file(path_of(dir, name, ".HashSeg_info"), hinfo) || !read_file(path_of(dir, name, ".segNum"), bnum) ||
        !read_file(path_of(dir, name, ".segOffset"), boff) ||
        !read_file(path_of(dir, name, ".ind2_distance_base"), base) ||
        !read_file(path_of(dir, name, ".regression_info"), reg))
        return EXCL_E_INVALID;
    const uint32_t nl = (uint32_t)ind1.size();
    const size_t nbk = boff.size();
    if (nl == 0 || hoff.size() != nl || bnum.size() != nl || base.size() != nbk || reg.size() != nbk)
        return EXCL_E_FORMAT;
    excl_index *ix = new (std::nothrow) excl_index();
    if (!ix) return EXCL_E_NOMEM;
    ix->nlists = nl;
    ix->lists.resize(nl);
    const uint64_t nwords = ind2.size();
    take_words(ix, ind2);
    ix->postings = 0;
    int st = EXCL_OK;
    std::vector<uint32_t> vals, docs, cnt;
    for (uint32_t l = 0; l < nl && !st; ++l) {
        const uint32_t n = ind1[l].length;
        const uint64_t wb = ind1[l].offset / 4;
        const uint64_t we = l + 1 < nl ? ind1[l + 1].offset / 4 : nwords;
        const size_t h = hoff[l];
        if (n == 0 || ind1[l].offset % 4 || wb > we || we > nwords || h + 2 > hinfo.size()) {
            st = EXCL_E_FORMAT;
            break;
        }
        const uint32_t shift = hinfo[h], nb = hinfo[h + 1];
        const size_t b0 = bnum[l];
        if (shift > 31 || nb == 0 || h + 3 + (size_t)nb > hinfo.size() || b0 > nbk || nb > nbk - b0 ||
            (l + 1 < nl && bnum[l + 1] != b0 + nb) || (l + 1 == nl && b0 + nb != nbk)) {
            st = EXCL_E_FORMAT;
            break;
        }
        const uint32_t *o = hinfo.data() + h + 2;  // element offsets of the buckets, nb + 1
        if (o[0] != 0 || o[nb] != n) {
            st = EXCL_E_FORMAT;
            break;
        }
        ListDesc &d = ix->lists[l];
        d.word_base = wb;
        d.n = n;
        d.seg_base = (uint32_t)ix->seg_head.size();
        d.codec = EXCL_CODEC_HS_SEGLRC;
        d.log2_block = 0;
        d.model = kNoModel;
        d.dir_shift = shift;
        d.ndir = nb;
        d.dir_base = (uint32_t)ix->dir.size();
        docs.assign(n, 0u);
        cnt.clear();
        uint32_t ns = 0;
        for (uint32_t b = 0; b < nb && !st; ++b) {
            ix->dir.push_back(ns);
            if (o[b + 1] < o[b]) {
                st = EXCL_E_FORMAT;
                break;
            }
            const uint32_t c = o[b + 1] - o[b];
            if (c == 0) continue;
            // this block ends where the next non-empty bucket's begins (or the list's words end)
            uint32_t nb2 = b + 1;
            while (nb2 < nb && o[nb2 + 1] == o[nb2]) ++nb2;
            const uint64_t ow = boff[b0 + b], next = nb2 < nb ? boff[b0 + nb2] : we - wb;
            const uint32_t *blk = ix->words.data() + wb + ow;
            if (ow >= next || wb + next > we || block_words(EXCL_CODEC_HS_SEGLRC, blk, c, next - ow) == ~0ull) {
                st = EXCL_E_FORMAT;
                break;
            }
            vals.resize(c);
            pfd_decode_block(blk, c, vals.data());
            const SegReg &rg = reg[b0 + b];
            for (uint32_t k = 0; k < c; ++k)
                docs[o[b] + k] = vals[k] + (uint32_t)seg_pred_host(k, rg.a, rg.b) + base[b0 + b];
            // every docID of the bucket hashes to it, and the list ascends
            for (uint32_t k = 0; k < c; ++k)
                if ((docs[o[b] + k] >> shift) != b || (o[b] + k && docs[o[b] + k] <= docs[o[b] + k - 1])) st = EXCL_E_FORMAT;
            if (st) break;
            ix->seg_head.push_back(docs[o[b]]);
            ix->seg_rec.push_back(SegRec{o[b], (uint32_t)ow, base[b0 + b], c});
            ix->seg_reg.push_back(rg);
            cnt.push_back(c);
            ++ns;
        }
        if (st) break;
        ix->dir.push_back(ns);
        d.nseg = ns;
        d.first_doc = docs[0];
        d.last_doc = docs[n - 1];
        if (d.last_doc >> shift != nb - 1) {
            st = EXCL_E_FORMAT;
            break;
        }
        // the list-level fit the builder keeps beside the buckets' fits
        const SegReg lf = fit_host(docs.data(), n);
        std::memcpy(d.reg, &lf, sizeof lf);
        d.tile_base = (uint32_t)ix->tilemap.size();
        if (variable_list_tiles(cnt.data(), ns, ix->tilemap)) {
            st = EXCL_E_FORMAT;
            break;
        }
        d.ntiles = (uint32_t)ix->tilemap.size() - d.tile_base;
        ix->postings += n;
    }
    if (st) {
        delete ix;
        return st;
    }
    *out = ix;
    return EXCL_OK;
}

}  // namespace

extern "C" int excl_index_save_reference(const excl_index *ix, const char *dir, const char *name) {
    if (!ix || !name || ix->nlists == 0) return EXCL_E_INVALID;
    const uint32_t codec = ix->lists[0].codec;
    if (!reference_codec(codec)) return EXCL_E_FORMAT;
    for (uint32_t l = 0; l < ix->nlists; ++l) {
        const ListDesc &d = ix->lists[l];
        // one codec; fixed formats in 256-entry segments
        if (d.codec != codec || (fixed_codec(codec) && d.log2_block != 8)) return EXCL_E_FORMAT;
    }
    if (codec == EXCL_CODEC_HS_SEGLRC) return save_hs(ix, dir, name);
    const size_t nsegs = ix->seg_head.size();
    const uint64_t nwords = ix->words.size() - kWordPad;
    const std::vector<Ind1> ind1 = ind1_of(ix);
    std::vector<uint32_t> seg_num(ix->nlists), seg_off(nsegs), aux(nsegs);
    for (uint32_t l = 0; l < ix->nlists; ++l) seg_num[l] = ix->lists[l].seg_base;
    for (size_t g = 0; g < nsegs; ++g) {
        seg_off[g] = ix->seg_rec[g].off;
        aux[g] = ix->seg_rec[g].aux;
    }
    bool ok = write_file(path_of(dir, name, ".ind1"), ind1.data(), ind1.size() * sizeof(Ind1)) &&
              write_file(path_of(dir, name, ".ind2"), ix->words.data(), nwords * 4) &&
              write_file(path_of(dir, name, ".segNum"), seg_num.data(), seg_num.size() * 4) &&
              write_file(path_of(dir, name, ".segHead"), ix->seg_head.data(), nsegs * 4) &&
              write_file(path_of(dir, name, ".segOffset"), seg_off.data(), nsegs * 4);
    std::vector<SegReg> list_reg(ix->nlists);
    for (uint32_t l = 0; l < ix->nlists; ++l) std::memcpy(&list_reg[l], ix->lists[l].reg, sizeof(SegReg));
    if (!ok) return EXCL_E_INVALID;
    switch (codec) {
        case EXCL_CODEC_PARAPFD:
        case EXCL_CODEC_NEWPFD:
            ok = write_file(path_of(dir, name, ".segMedian"), aux.data(), nsegs * 4);
            break;
        case EXCL_CODEC_SEGLRC:
            ok = write_file(path_of(dir, name, ".ind2_distance_base"), aux.data(), nsegs * 4) &&
                 write_file(path_of(dir, name, ".regression_info"), ix->seg_reg.data(), nsegs * sizeof(SegReg)) &&
                 write_file(path_of(dir, name, ".regression_info_list"), list_reg.data(),
                            list_reg.size() * sizeof(SegReg));
            break;
        case EXCL_CODEC_LRCSEG:
            ok = write_file(path_of(dir, name, ".ind2_distance_base"), aux.data(), nsegs * 4) &&
                 write_file(path_of(dir, name, ".regression_info"), list_reg.data(), list_reg.size() * sizeof(SegReg));
            break;
        default: {  // LRC
            std::vector<LrcReg> lr(ix->nlists);
            for (uint32_t l = 0; l < ix->nlists; ++l) std::memcpy(&lr[l], ix->lists[l].reg, sizeof(LrcReg));
            ok = write_file(path_of(dir, name, ".regression_info"), lr.data(), lr.size() * sizeof(LrcReg));
        }
    }
    return ok ? EXCL_OK : EXCL_E_INVALID;
}

extern "C" int excl_index_load_reference(const char *dir, const char *name, uint32_t codec, excl_index **out) {
    if (!name || !out || !reference_codec(codec)) return EXCL_E_INVALID;
    *out = nullptr;
    if (codec == EXCL_CODEC_HS_SEGLRC) return load_hs(dir, name, out);
    const bool dgap = codec_is_dgap(codec);
    std::vector<Ind1> ind1;
    std::vector<uint32_t> ind2, seg_num, seg_head, seg_off, aux;
    std::vector<SegReg> reg, list_reg;
    std::vector<LrcReg> lrc_reg;
    if (!read_file(path_of(dir, name, ".ind1"), ind1) || !read_file(path_of(dir, name, ".ind2"), ind2) ||
        !read_file(path_of(dir, name, ".segNum"), seg_num) || !read_file(path_of(dir, name, ".segHead"), seg_head) ||
        !read_file(path_of(dir, name, ".segOffset"), seg_off))
        return EXCL_E_INVALID;
    bool ok = true;
    if (dgap) ok = read_file(path_of(dir, name, ".segMedian"), aux);
    else if (codec == EXCL_CODEC_SEGLRC)
        ok = read_file(path_of(dir, name, ".ind2_distance_base"), aux) &&
             read_file(path_of(dir, name, ".regression_info"), reg) &&
             read_file(path_of(dir, name, ".regression_info_list"), list_reg);
    else if (codec == EXCL_CODEC_LRCSEG)
        ok = read_file(path_of(dir, name, ".ind2_distance_base"), aux) &&
             read_file(path_of(dir, name, ".regression_info"), list_reg);
    else
        ok = read_file(path_of(dir, name, ".regression_info"), lrc_reg);
    if (!ok) return EXCL_E_INVALID;
    const uint32_t nl = (uint32_t)ind1.size();
    const size_t ns = seg_head.size();
    if (codec == EXCL_CODEC_LRC) aux.assign(ns, 0u);  // no per-segment base
    if (nl == 0 || seg_num.size() != nl || seg_off.size() != ns || aux.size() != ns ||
        (codec == EXCL_CODEC_SEGLRC && reg.size() != ns) ||
        ((codec == EXCL_CODEC_SEGLRC || codec == EXCL_CODEC_LRCSEG) && list_reg.size() != nl) ||
        (codec == EXCL_CODEC_LRC && lrc_reg.size() != nl))
        return EXCL_E_FORMAT;
    excl_index *ix = new (std::nothrow) excl_index();
    if (!ix) return EXCL_E_NOMEM;
    ix->nlists = nl;
    ix->lists.resize(nl);
    const uint64_t nwords = ind2.size();
    take_words(ix, ind2);
    ix->seg_head = std::move(seg_head);
    ix->seg_rec.resize(ns);
    ix->seg_reg.assign(ns, SegReg{1.0f, 0.0f, 0, 0});
    ix->postings = 0;
    int st = EXCL_OK;
    std::vector<uint32_t> vals(kRefSegment), ldir;
    for (uint32_t l = 0; l < nl && !st; ++l) {
        const uint32_t n = ind1[l].length;
        const uint32_t nseg = (n + kRefSegment - 1) / kRefSegment;
        const uint64_t wb = ind1[l].offset / 4;
        // the list's words end where the next list's begin (or at the end of .ind2)
        const uint64_t we = l + 1 < nl ? ind1[l + 1].offset / 4 : nwords;
        if (n == 0 || ind1[l].offset % 4 || wb > we || we > nwords || seg_num[l] > ns || nseg > ns - seg_num[l] ||
            (l + 1 < nl && seg_num[l + 1] != seg_num[l] + nseg) || (l + 1 == nl && seg_num[l] + nseg != ns)) {
            st = EXCL_E_FORMAT;
            break;
        }
        ListDesc &d = ix->lists[l];
        d.word_base = wb;
        d.n = n;
        d.seg_base = seg_num[l];
        d.nseg = nseg;
        d.codec = codec;
        d.log2_block = 8;
        d.model = kNoModel;
        d.first_doc = ix->seg_head[d.seg_base];
        if (codec == EXCL_CODEC_SEGLRC || codec == EXCL_CODEC_LRCSEG) std::memcpy(d.reg, &list_reg[l], sizeof(SegReg));
        if (codec == EXCL_CODEC_LRC) std::memcpy(d.reg, &lrc_reg[l], sizeof(LrcReg));
        for (uint32_t s = 0; s < nseg; ++s) {
            const size_t g = (size_t)d.seg_base + s;
            const uint32_t cnt = std::min(kRefSegment, n - s * kRefSegment);
            const uint64_t ow = seg_off[g];
            const uint64_t next = s + 1 < nseg ? seg_off[g + 1] : we - wb;
            // the block must lie inside the list's words and decode within itself
            const uint32_t *blk = ix->words.data() + wb + ow;
            if (ow >= next || wb + next > we || (s && ix->seg_head[g] <= ix->seg_head[g - 1]) ||
                block_words(codec, blk, cnt, next - ow) == ~0ull) {
                st = EXCL_E_FORMAT;
                break;
            }
            SegRec &r = ix->seg_rec[g];
            r.start = s * kRefSegment;
            r.off = (uint32_t)ow;
            r.aux = aux[g];
            r.count = cnt;
            if (codec == EXCL_CODEC_SEGLRC) ix->seg_reg[g] = reg[g];
        }
        if (st) break;
        // last docID: decode the list's last block
        const size_t gl = (size_t)d.seg_base + nseg - 1;
        const SegRec &rl = ix->seg_rec[gl];
        const uint32_t *blk = ix->words.data() + wb + rl.off;
        if (codec == EXCL_CODEC_NEWPFD) newpfd_decode_block(blk, rl.count, vals.data());
        else pfd_decode_block(blk, rl.count, vals.data());
        const uint32_t t = rl.count - 1, i = rl.start + t;  // the last value: index in its segment and list
        float a, b;
        std::memcpy(&a, &d.reg[0], 4);
        std::memcpy(&b, &d.reg[1], 4);
        if (dgap) {
            uint32_t v = ix->seg_head[gl];
            for (uint32_t k = 1; k < rl.count; ++k) v += vals[k];
            d.last_doc = v;
        } else if (codec == EXCL_CODEC_SEGLRC) {
            const SegReg &rg = ix->seg_reg[gl];
            d.last_doc = vals[t] + (uint32_t)seg_pred_host(t, rg.a, rg.b) + rl.aux;
        } else if (codec == EXCL_CODEC_LRCSEG) {
            d.last_doc = vals[t] + (uint32_t)seg_pred_host(i, a, b) + rl.aux;
        } else {
            d.last_doc = vals[t] + lrc_pred_host(i, a, (int32_t)d.reg[1]);
        }
        if (d.last_doc < d.first_doc) {
            st = EXCL_E_FORMAT;
            break;
        }
        fixed_list_directory(d, ix->seg_head.data() + d.seg_base, nseg, ldir);
        d.dir_base = (uint32_t)ix->dir.size();
        ix->dir.insert(ix->dir.end(), ldir.begin(), ldir.end());
        d.tile_base = 0;
        d.ntiles = nseg;
        ix->postings += n;
    }
    if (st) {
        delete ix;
        return st;
    }
    *out = ix;
    return EXCL_OK;
}

extern "C" int excl_query_parse(const void *buf, size_t bytes, uint32_t *terms, size_t terms_cap,
                                uint32_t *term_offsets, size_t queries_cap, uint32_t *nq_out, size_t *nterms_out) {
    if ((!buf && bytes) || !nq_out || !nterms_out || bytes % 4) return EXCL_E_INVALID;
    const uint32_t *w = static_cast<const uint32_t *>(buf);
    const size_t nw = bytes / 4;
    size_t i = 0, nt = 0;
    uint32_t nq = 0;
    int st = EXCL_OK;
    while (i < nw) {
        const uint32_t k = w[i++];
        if (k > kMaxTerms || k > nw - i) return EXCL_E_FORMAT;
        if (term_offsets && nq < queries_cap) term_offsets[nq] = (uint32_t)nt;
        else if (term_offsets) st = EXCL_E_CAPACITY;
        for (uint32_t j = 0; j < k; ++j, ++nt) {
            if (terms && nt < terms_cap) terms[nt] = w[i + j];
            else if (terms) st = EXCL_E_CAPACITY;
        }
        i += k;
        ++nq;
    }
    if (term_offsets && nq < queries_cap) term_offsets[nq] = (uint32_t)nt;
    else if (term_offsets) st = EXCL_E_CAPACITY;
    *nq_out = nq;
    *nterms_out = nt;
    return st;
}

extern "C" int excl_query_encode(const uint32_t *terms, const uint32_t *term_offsets, uint32_t nq, void *buf,
                                 size_t cap, size_t *bytes) {
    if (!term_offsets || !bytes) return EXCL_E_INVALID;
    size_t need = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        if (term_offsets[q + 1] < term_offsets[q]) return EXCL_E_INVALID;
        need += 4 * (1 + (size_t)(term_offsets[q + 1] - term_offsets[q]));
    }
    *bytes = need;
    if (!buf) return EXCL_OK;
    if (need > cap) return EXCL_E_CAPACITY;
    uint32_t *w = static_cast<uint32_t *>(buf);
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t k = term_offsets[q + 1] - term_offsets[q];
        *w++ = k;
        if (k) std::memcpy(w, terms + term_offsets[q], (size_t)k * 4);
        w += k;
    }
    return EXCL_OK;
}
