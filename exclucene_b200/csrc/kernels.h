// The per-batch device view and the launchers of kernels.cu / decode.cu.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>

#include "excl_device.cuh"

namespace excl {

struct BatchView {
    uint32_t nq;
    const uint32_t *qterms;      // nq * kMaxTerms list ids, ascending length
    const uint32_t *qnterms;     // terms per query
    const uint32_t *tile_prefix; // nq + 1, exclusive prefix of tiles per query
    uint32_t *tile_q;            // max_tiles: query + 1 where the tile is its query's first tile, else 0;
                                 // then (scatter phase) the tile's output position
    uint4 *tile_order;           // max_tiles work records {tile, query, tile within the query, shortest list}:
                                 // heavy tiles from the front, the rest from the back (tile_prefix[nq + 1] = heavy tiles)
    uint32_t *tile_counter;      // work-queue head (zeroed by the pack phase)
    const uint32_t *key_base;    // nq + 1, exclusive prefix of shortest-list lengths
    uint32_t *tile_count;        // survivors per tile
    uint32_t *tile_slot;         // scratch position of each tile's survivors
    uint32_t *scratch;           // max_keys survivor slots, indexed by key position
    uint32_t max_tiles;
    uint32_t merge_segs;         // probe: merge when a tile's keys span at most this many segments (0: never)
    uint32_t tile_split;         // fixed-block shortest lists: each segment is cut into 2^tile_split tiles
    uint64_t max_keys;
    uint32_t *err;               // error flag bits
    uint32_t *err_out;           // or null: device-mapped host word that receives this batch's error bits at its end (the device word is cleared)
    uint32_t *probe_done;        // tiles probed so far (cleared by the pack phase)
    uint32_t *scatter_ready;     // scatter chunks whose output positions are out (cleared by the pack phase)
    uint32_t check_polls;        // > 0: one bounded wait on check_flag (which nothing sets) that must give up
    const uint32_t *check_flag;
    uint64_t *stats;             // or null: [probes, fallbacks, keys, merges, t_start, t_packed, t_probed, t_end]
                                 // (times in globaltimer ns)
};

// probe phase: shared-memory merge of a tile's keys against a decoded span
constexpr uint32_t kMergeCap = 512;      // docIDs of the span (two 256-blocks)
constexpr uint32_t kMergeMinKeys = 32;   // fewer keys than this: always probe

// the batch kernel's phases (kernels.cu, batch_phases.cuh)
constexpr uint32_t kPackThreads = 256;
constexpr uint32_t kPackMaxCtas = 1024;
constexpr uint32_t kPackMaxQueries = kPackThreads * kPackMaxCtas;
constexpr uint32_t kSSThreads = 256;
constexpr uint32_t kSSChunk = 512;
constexpr uint32_t kBatchWarps = 8;  // warps per CTA of the batch kernel (every phase)

// Cross-CTA state of one stream's batches (zeroed once at allocation; the
// kernels tag what they publish with the batch, so it is never cleared).
struct PackSync {
    uint32_t epoch;           // tag of the last batch run on this state
    uint32_t ticket;          // pack phase: chunk tickets
    uint32_t sticket, sdone;  // scatter phase: chunk tickets; CTAs that left the kernel
    uint32_t flag[kPackMaxCtas];  // pack chunk c: tag << 1 once its aggregates are out
    uint32_t agg_t[kPackMaxCtas];
    uint32_t agg_k[kPackMaxCtas];
    uint32_t agg_h[kPackMaxCtas];
    // pack chunks whose writes are all visible (the probe phase starts when it
    // reaches the batch's chunks; reset by the last CTA out). Every CTA polls
    // it, so it has a cache line of its own.
    alignas(128) uint32_t packed;
};

// Queries per pack chunk: small chunks spread the pack's gathers (terms,
// list descriptors) over many SMs; larger ones keep big batches within the
// kPackMaxCtas chunk slots.
__host__ __device__ inline uint32_t pack_chunk_queries(uint32_t nq) {
    return nq <= 64u * kPackMaxCtas ? 64u : (nq <= 128u * kPackMaxCtas ? 128u : 256u);
}

// Everything one batch launch needs.
struct BatchLaunch {
    DevIndexView ixv;
    const ListDesc *lists;
    uint32_t nlists;
    const uint32_t *terms, *toff;  // the batch's queries (device or host-mapped)
    BatchView b;
    PackSync *sync;
    uint64_t *chunk_state;  // max_tiles / kSSChunk + 1 words
    uint32_t *offsets;      // nq + 1
    uint32_t *docids;       // cap
    uint64_t cap;
    int algo, warps, ctas_per_sm, nsm;
    uint32_t max_ctas;  // > 0: launch at most this many CTAs (a batch whose tile count the host knows needs
                        // no more than one warp per tile); 0: every CTA that fits on the device
    uint32_t spin;    // polls before a cross-CTA wait gives up (0: the default)
    cudaEvent_t *ev;  // 4 events around the batch kernel, or null
};

// The batch kernel (pack, probe, scatter in one launch) on `st`.
int launch_batch(const BatchLaunch &L, cudaStream_t st);

// tk: two zeroed words (work counter, finished CTAs), left zeroed.
int launch_decode(const DevIndexView &ix, uint32_t l0, uint32_t l1, uint64_t out_base0, uint32_t *out, uint32_t seg0,
                  uint32_t nsegs, int nsm, uint32_t *tk, uint32_t *err, cudaStream_t st);

}  // namespace excl
