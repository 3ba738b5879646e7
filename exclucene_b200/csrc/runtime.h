// Host-side state of a context and of a device-resident index.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "excl_device.cuh"
#include "kernels.h"

namespace excl {

struct DeviceIndex {
    ListDesc *lists = nullptr;
    uint32_t *words = nullptr;
    uint32_t *seg_head = nullptr;
    SegRec *seg_rec = nullptr;
    SegReg *seg_reg = nullptr;
    uint32_t *dir = nullptr;
    uint64_t *tilemap = nullptr;
    uint64_t *post_base = nullptr;
    uint32_t *seg_list = nullptr;
    uint64_t *seg_gword = nullptr;
    ProbeRec *seg_probe = nullptr;
    uint32_t codec_mask = 0;  // bit c: some list has codec c
    size_t bytes = 0;
    int device = 0;
    void release();
    DevIndexView view(const ModelView &mv) const;
};

// slots of ctx->d_misc
enum {
    kMiscErr = 0,
    kMiscTileCounter = 1,
    kMiscDecodeTicket = 2,  // and 3: decode work counter, CTAs done
    kMiscNeverSet = 5,      // stays 0: the flag of the failure-path self-test wait
    kMiscProbeDone = 32,    // tiles probed (batch kernel); its own 128-byte line, apart from the queue head
    kMiscScatterReady = 48, // scatter chunks ready (batch kernel); another line
    kMiscWords = 64,
};
// excl_submit_into batches that may be in flight on one context at once
constexpr uint32_t kFlagSlots = 256;

}  // namespace excl

struct excl_ctx {
    int device = 0;
    int nsm = 148;
    int warps = 8;
    int ctas_per_sm = 4;
    uint32_t merge_segs = 2;
    uint32_t tile_split = 0;  // log2 of the tiles each fixed segment of a shortest list is cut into
    int tuned_algo = -1;  // search method the autotuner chose for EXCL_ALGO_AUTO (-1: none)
    bool collect_stats = true;
    uint32_t spin_limit = 0;  // polls before a cross-CTA wait of the batch kernel gives up (0: the default)
    uint32_t wait_check_polls = 0;  // excl_ctx_set_wait_check
    // CUDA graph of the last batch launched through excl_intersect_device
    bool use_graphs = false, last_was_graph = false;
    cudaGraphExec_t gexec = nullptr;
    uint64_t gkey[12] = {};
    bool gkey_seen = false;  // the key ran once uncaptured (first sighting)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    excl_ctx_config cfg{};
    std::mutex mu;
    std::string last_error;
    uint32_t max_tiles = 0;
    uint32_t last_nq = 0;
    uint32_t *d_terms = nullptr, *d_toff = nullptr;
    uint32_t *d_qterms = nullptr, *d_qnterms = nullptr, *d_tile_prefix = nullptr, *d_tile_q = nullptr;
    uint32_t *d_tile_count = nullptr, *d_scratch = nullptr, *d_misc = nullptr;
    uint32_t *d_key_base = nullptr, *d_tile_slot = nullptr;
    uint4 *d_tile_order = nullptr;
    excl::PackSync *d_sync = nullptr;
    uint64_t *d_stats = nullptr, *d_chunk_state = nullptr;
    uint32_t *d_offsets = nullptr, *d_docids = nullptr;
    uint64_t docids_cap = 0;
    uint32_t *h_terms = nullptr, *h_toff = nullptr, *h_offsets = nullptr;
    // error word of each batch in flight (pinned, device-mapped: the scatter
    // kernel writes it) and the event that marks the batch done, a slot per batch
    uint32_t *h_flags = nullptr, *m_flags = nullptr;
    cudaEvent_t slot_ev[excl::kFlagSlots] = {};
    std::vector<uint32_t> free_flag_slots;
    // Entry points that use the context's stream, buffers or settings hold
    // this lock, so host threads may share a context; excl_wait holds it only
    // to copy an excl_submit batch's results, never while waiting.
    std::recursive_mutex op_mu;
    uint64_t submit_seq = 0;  // excl_submit batches so far (their results share the context's buffers)
};

namespace excl {
void ctx_error(excl_ctx *ctx, const char *fmt, ...);
int cuda_status(excl_ctx *ctx, cudaError_t e, const char *what);
int read_device_flags(excl_ctx *ctx);
int flags_status(excl_ctx *ctx, uint32_t f);
// tiles_hint > 0: the batch's tile count, known on the host, caps the grid at one warp per tile
int run_pipeline(excl_ctx *ctx, excl_index *ix, const uint32_t *d_terms, const uint32_t *d_toff, uint32_t nq,
                 uint32_t algo, uint32_t *d_offsets, uint32_t *d_docids, uint64_t cap, uint32_t *err_out = nullptr,
                 uint32_t tiles_hint = 0);
// Tiles of a batch of at most kHostTilesMaxQueries queries whose terms are in
// host memory (the shortest list's tiles per query, as the pack phase counts
// them); 0 for larger batches, which take the whole device anyway.
constexpr uint32_t kHostTilesMaxQueries = 512;
uint32_t host_batch_tiles(const excl_ctx *ctx, const excl_index *ix, const uint32_t *terms,
                          const uint32_t *term_offsets, uint32_t nq);

// learned.cu
ModelView model_view(const ModelSet *m);
int models_upload(excl_ctx *ctx, excl_index *ix);
void models_free(ModelSet *m);
}  // namespace excl
