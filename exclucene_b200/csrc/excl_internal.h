// Internal layout shared by the host builder (codec.cpp) and the device
// kernels (*.cu). Not part of the C ABI.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/excl_gpu.h"

namespace excl {

constexpr uint32_t kNoModel = 0xffffffffu;
constexpr uint32_t kMaxTerms = 32;    // terms per query on the device
constexpr uint32_t kTileKeys = 256;   // keys per tile (one shortest-list segment or a 256-slice of an HS bucket)
constexpr uint32_t kWordPad = 8;      // zero words after the last block: 64/128-bit window reads stay in bounds
constexpr uint32_t kMinBlock = 32;    // smallest fixed block (bounds tiles per key for buffer sizing)

// Tile map entry of a variable-segment (HS) list: first segment of the tile
// (within the list), first element within that segment, number of segments.
constexpr uint32_t kTileMaxE0 = (1u << 24) - 1;
constexpr uint32_t kTileMaxSegs = 255;
inline constexpr uint64_t tile_pack(uint32_t seg, uint32_t e0, uint32_t nseg) {
    return ((uint64_t)seg << 32) | ((uint64_t)e0 << 8) | nseg;
}

// Device-resident description of one posting list (80 bytes, 16-byte aligned
// so a warp reads it with 128-bit loads). The first 16 bytes hold what the
// batch kernel's pack phase reads per query term (length, tiles, block size),
// so that costs one vector load.
struct alignas(16) ListDesc {
    uint32_t n;           // postings
    uint32_t ntiles;      // tiles when this list is the shortest of a query
    uint32_t log2_block;  // fixed block size = 1 << log2_block; 0 = variable (HS)
    uint32_t seg_base;    // first segment of the list in the per-segment arrays
    uint64_t word_base;   // first word of the list's blocks in the words[] array
    uint32_t nseg;        // segments (fixed blocks, or non-empty HS blocks)
    uint32_t codec;       // excl_codec
    uint32_t first_doc;
    uint32_t last_doc;
    uint32_t reg[4];      // list-level regression raw bits (LRC: slope, icpt, range, 0; others a, b, L, R)
    uint32_t dir_shift;   // bucket = docID >> dir_shift
    uint32_t dir_base;    // first directory entry (ndir + 1 entries)
    uint32_t ndir;        // buckets
    uint32_t tile_base;   // variable lists: first tilemap entry
    uint32_t model;       // learned model slot or kNoModel
    uint32_t pad;
};
static_assert(sizeof(ListDesc) == 80, "ListDesc layout");
static_assert(offsetof(ListDesc, n) == 0 && offsetof(ListDesc, ntiles) == 4 && offsetof(ListDesc, log2_block) == 8,
              "the pack phase reads n, ntiles and log2_block as one 16-byte vector");

// Per-segment record: start element, word offset within the list, aux
// (ParaPFD: docID at the segment middle = segMedian; residual codecs: base).
struct alignas(16) SegRec {
    uint32_t start;
    uint32_t off;
    uint32_t aux;
    uint32_t count;
};

struct alignas(16) SegReg {
    float a;
    float b;
    uint32_t L;
    uint32_t R;
};

// Everything a probe needs about one segment, in one 64-byte record built at
// upload; the first 32 bytes serve a plain probe of any codec, so the
// segment search, the record and the block header cost one memory round trip.
constexpr uint32_t kProbeUnbounded = 0xffffu;  // window range too wide for 16 bits
struct alignas(64) ProbeRec {
    uint32_t head;   // first docID (seg_head)
    uint32_t off;    // block's word offset within the list
    uint32_t aux;    // SegRec.aux
    uint32_t count;  // elements
    uint32_t hdr;    // the block's descriptor word
    float a, b;      // segment regression (SegLRC, HS_SegLRC)
    uint32_t lr;     // regression window ranges L | R << 16, kProbeUnbounded if wider
    uint32_t start;  // list position of the first element (second half: HS lists only)
    // whole-list decode: the list's codec and regression words, the segment's
    // first output position, so a decode plan needs no second dependent load
    uint32_t codec;
    uint64_t ob;
    uint32_t r0, r1;
    uint32_t pad[2];
};
static_assert(sizeof(ProbeRec) == 64, "ProbeRec layout");
static_assert(offsetof(ProbeRec, a) == 20 && offsetof(ProbeRec, start) == 32 && offsetof(ProbeRec, codec) == 36 &&
                  offsetof(ProbeRec, ob) == 40 && offsetof(ProbeRec, r0) == 48,
              "decode plans read ProbeRec as four 16-byte vectors");

#ifdef __CUDACC__
#define EXCL_HD __host__ __device__ __forceinline__
#else
#define EXCL_HD inline
#endif

EXCL_HD bool codec_is_hs(uint32_t c) { return c == EXCL_CODEC_HS_SEGLRC || c == EXCL_CODEC_HS_PARAPFD; }
EXCL_HD bool codec_is_dgap(uint32_t c) {
    return c == EXCL_CODEC_PARAPFD || c == EXCL_CODEC_HS_PARAPFD || c == EXCL_CODEC_NEWPFD;
}
EXCL_HD bool codec_is_newpfd(uint32_t c) { return c == EXCL_CODEC_NEWPFD; }

struct DeviceIndex;  // runtime.cu
struct ModelSet;     // learned.cu

// Host image of a built index.
struct HostIndex {
    uint32_t nlists = 0;
    uint64_t postings = 0;
    std::vector<ListDesc> lists;
    std::vector<uint32_t> words;
    std::vector<uint32_t> seg_head;
    std::vector<SegRec> seg_rec;
    std::vector<SegReg> seg_reg;
    std::vector<uint32_t> dir;
    std::vector<uint64_t> tilemap;   // (segment within list << 32) | first element within segment
    DeviceIndex *dev = nullptr;
    ModelSet *models = nullptr;
};

// codec.cpp
uint32_t pfd_encode_block(const uint32_t *in, uint32_t n, float frac, uint32_t *out, int *err);
uint32_t pfd_decode_block(const uint32_t *in, uint32_t n, uint32_t *out);
uint32_t pfd_block_words(const uint32_t *in, uint32_t n);
uint32_t newpfd_encode_block(const uint32_t *in, uint32_t n, float frac, uint32_t *out, int *err);
uint32_t newpfd_decode_block(const uint32_t *in, uint32_t n, uint32_t *out);
// Words of a NewPFD block, found by walking its Simple-16 selectors without
// reading past `avail` words (~0 if the block does not fit in them).
uint64_t newpfd_block_words(const uint32_t *in, uint32_t n, uint64_t avail);
int build_index(const uint32_t *docs, const uint64_t *loff, uint32_t nlists, const excl_build_params &p,
                HostIndex &ix, std::string &err);
// Top-bits directory of a fixed-block list (about one segment per bucket);
// sets d.dir_shift / d.ndir from d.last_doc.
void fixed_list_directory(ListDesc &d, const uint32_t *head, uint32_t ns, std::vector<uint32_t> &dir);
// SegLRC/LRCSeg/HS prediction (int)(idx * a + b) with one rounding, saturating.
int32_t seg_pred_host(uint32_t idx, float a, float b);
// LRC prediction (int)((float)i * slope) + icpt (LRC_Generator_kernel.cu:70), wrapping.
uint32_t lrc_pred_host(uint32_t idx, float slope, int32_t icpt);
// Tile map of a variable-segment (HS) list from its segment counts.
int variable_list_tiles(const uint32_t *cnt, uint32_t ns, std::vector<uint64_t> &tiles);
// The least-squares fit of SegLRC/LRCSeg (segment or list level) on the host.
SegReg fit_host(const uint32_t *y, uint32_t n);
// The LRC list fit on the host (LRC_Generator.cu:221-287): slope, intercept, range.
void fit_lrc_host(const uint32_t *y, uint32_t n, float *slope, int32_t *icpt, float *range);

}  // namespace excl

struct excl_index : excl::HostIndex {};
