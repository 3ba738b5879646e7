// The reference's on-disk index and query files, read and written as they are,
// so an index produced by its encoders runs here unchanged and an index built
// here can be handed to its binaries.
//
// File sets (`<dir>/<name><suffix>`; the reference keeps the regression files
// in a second directory, here they sit beside the others):
//
//   ParaPFD (ParaPFD_Compression/main.cpp:81-232, SegmentSize 256)
//     .ind1        per list {u32 length; u64 byte offset into .ind2}, 16 bytes
//                  with the x86-64 padding after length (main.cpp:32-35)
//     .ind2        the lists' ParaPFD blocks, list after list
//     .segNum      u32 per list: index of its first segment
//     .segHead     u32 per segment: its first docID
//     .segMedian   u32 per segment: docID at count / 2
//     .segOffset   u32 per segment: word offset of its block within the list
//   SegLRC (SegLRC_Compression/main.cpp:80-207, SegLRC_Generator.cu:94-436)
//     .ind1 .ind2 .segNum .segHead .segOffset as above (blocks of residuals)
//     .ind2_distance_base     i32 per segment: the residuals' minimum
//     .regression_info        per segment {float a; float b; u32 L; u32 R}
//     .regression_info_list   per list, same record (list-level fit)
//   Queries (ParaPFD_Intersection.cu:139-142)
//     .query       per query u32 term count, then that many u32 term ids
//
// The layout of these arrays is the layout of this library's index (lists and
// segments in the same order, the same block bytes, word offsets within the
// list), so loading copies them and derives the rest (segment counts and
// starts, last docIDs, directories).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "excl_internal.h"

using namespace excl;

namespace {

constexpr uint32_t kRefSegment = 256;  // SegmentSize of the reference encoders

struct Ind1 {
    uint32_t length;
    uint32_t pad;
    uint64_t offset;
};
static_assert(sizeof(Ind1) == 16, "the reference's at_term_ind1_t is 16 bytes");

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

bool reference_codec(uint32_t c) {
    return c == EXCL_CODEC_PARAPFD || c == EXCL_CODEC_SEGLRC || c == EXCL_CODEC_NEWPFD;
}

}  // namespace

extern "C" int excl_index_save_reference(const excl_index *ix, const char *dir, const char *name) {
    if (!ix || !name || ix->nlists == 0) return EXCL_E_INVALID;
    const uint32_t codec = ix->lists[0].codec;
    if (!reference_codec(codec)) return EXCL_E_FORMAT;
    for (uint32_t l = 0; l < ix->nlists; ++l) {
        const ListDesc &d = ix->lists[l];
        if (d.codec != codec || d.log2_block != 8) return EXCL_E_FORMAT;  // one codec, 256-entry segments
    }
    const size_t nsegs = ix->seg_head.size();
    const uint64_t nwords = ix->words.size() - kWordPad;
    std::vector<Ind1> ind1(ix->nlists);
    std::vector<uint32_t> seg_num(ix->nlists), seg_off(nsegs), aux(nsegs);
    for (uint32_t l = 0; l < ix->nlists; ++l) {
        const ListDesc &d = ix->lists[l];
        ind1[l] = Ind1{d.n, 0u, d.word_base * 4};
        seg_num[l] = d.seg_base;
    }
    for (size_t g = 0; g < nsegs; ++g) {
        seg_off[g] = ix->seg_rec[g].off;
        aux[g] = ix->seg_rec[g].aux;
    }
    bool ok = write_file(path_of(dir, name, ".ind1"), ind1.data(), ind1.size() * sizeof(Ind1)) &&
              write_file(path_of(dir, name, ".ind2"), ix->words.data(), nwords * 4) &&
              write_file(path_of(dir, name, ".segNum"), seg_num.data(), seg_num.size() * 4) &&
              write_file(path_of(dir, name, ".segHead"), ix->seg_head.data(), nsegs * 4) &&
              write_file(path_of(dir, name, ".segOffset"), seg_off.data(), nsegs * 4);
    if (ok && codec != EXCL_CODEC_SEGLRC) {
        ok = write_file(path_of(dir, name, ".segMedian"), aux.data(), nsegs * 4);
    } else if (ok) {
        std::vector<SegReg> list_reg(ix->nlists);
        for (uint32_t l = 0; l < ix->nlists; ++l) std::memcpy(&list_reg[l], ix->lists[l].reg, sizeof(SegReg));
        ok = write_file(path_of(dir, name, ".ind2_distance_base"), aux.data(), nsegs * 4) &&
             write_file(path_of(dir, name, ".regression_info"), ix->seg_reg.data(), nsegs * sizeof(SegReg)) &&
             write_file(path_of(dir, name, ".regression_info_list"), list_reg.data(),
                        list_reg.size() * sizeof(SegReg));
    }
    return ok ? EXCL_OK : EXCL_E_INVALID;
}

extern "C" int excl_index_load_reference(const char *dir, const char *name, uint32_t codec, excl_index **out) {
    if (!name || !out || !reference_codec(codec)) return EXCL_E_INVALID;
    *out = nullptr;
    std::vector<Ind1> ind1;
    std::vector<uint32_t> ind2, seg_num, seg_head, seg_off, aux;
    std::vector<SegReg> reg, list_reg;
    if (!read_file(path_of(dir, name, ".ind1"), ind1) || !read_file(path_of(dir, name, ".ind2"), ind2) ||
        !read_file(path_of(dir, name, ".segNum"), seg_num) || !read_file(path_of(dir, name, ".segHead"), seg_head) ||
        !read_file(path_of(dir, name, ".segOffset"), seg_off))
        return EXCL_E_INVALID;
    if (codec != EXCL_CODEC_SEGLRC) {
        if (!read_file(path_of(dir, name, ".segMedian"), aux)) return EXCL_E_INVALID;
    } else if (!read_file(path_of(dir, name, ".ind2_distance_base"), aux) ||
               !read_file(path_of(dir, name, ".regression_info"), reg) ||
               !read_file(path_of(dir, name, ".regression_info_list"), list_reg)) {
        return EXCL_E_INVALID;
    }
    const uint32_t nl = (uint32_t)ind1.size();
    const size_t ns = seg_head.size();
    if (nl == 0 || seg_num.size() != nl || seg_off.size() != ns || aux.size() != ns ||
        (codec == EXCL_CODEC_SEGLRC && (reg.size() != ns || list_reg.size() != nl)))
        return EXCL_E_FORMAT;
    excl_index *ix = new (std::nothrow) excl_index();
    if (!ix) return EXCL_E_NOMEM;
    ix->nlists = nl;
    ix->lists.resize(nl);
    ix->words = std::move(ind2);
    const uint64_t nwords = ix->words.size();
    ix->words.resize(nwords + kWordPad, 0u);
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
        if (codec == EXCL_CODEC_SEGLRC) std::memcpy(d.reg, &list_reg[l], sizeof(SegReg));
        for (uint32_t s = 0; s < nseg; ++s) {
            const size_t g = (size_t)d.seg_base + s;
            const uint32_t cnt = std::min(kRefSegment, n - s * kRefSegment);
            const uint64_t ow = seg_off[g];
            const uint64_t next = s + 1 < nseg ? seg_off[g + 1] : we - wb;
            // the block must lie inside the list's words and decode within itself
            const uint32_t *blk = ix->words.data() + wb + ow;
            const uint64_t bw = codec == EXCL_CODEC_NEWPFD ? newpfd_block_words(blk, cnt, next - ow)
                                                           : pfd_block_words(blk, cnt);
            if (ow >= next || wb + next > we || (s && ix->seg_head[g] <= ix->seg_head[g - 1]) || bw > next - ow) {
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
        if (codec == EXCL_CODEC_NEWPFD) newpfd_decode_block(ix->words.data() + wb + rl.off, rl.count, vals.data());
        else pfd_decode_block(ix->words.data() + wb + rl.off, rl.count, vals.data());
        if (codec != EXCL_CODEC_SEGLRC) {
            uint32_t v = ix->seg_head[gl];
            for (uint32_t k = 1; k < rl.count; ++k) v += vals[k];
            d.last_doc = v;
        } else {
            const SegReg &rg = ix->seg_reg[gl];
            d.last_doc = vals[rl.count - 1] + (uint32_t)seg_pred_host(rl.count - 1, rg.a, rg.b) + rl.aux;
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
