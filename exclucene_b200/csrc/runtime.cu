// C ABI of libexcl_gpu.so: codec calls, index build/upload, contexts, the
// batched query pipeline and its host-buffer submit/wait form.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "excl_device.cuh"
#include "kernels.h"
#include "runtime.h"

using namespace excl;

// ---------------------------------------------------------------------------
// Codec calls.

extern "C" int excl_parapfd_encode(const uint32_t *in, uint32_t n, float frac, uint32_t *out, size_t cap,
                                   size_t *words) {
    if ((!in && n) || !out || !words) return EXCL_E_INVALID;
    std::vector<uint32_t> tmp((size_t)n * 3 + 8);
    int err = 0;
    const uint32_t w = pfd_encode_block(in, n, frac, tmp.data(), &err);
    if (err) return err;
    if (w > cap) return EXCL_E_CAPACITY;
    std::memcpy(out, tmp.data(), (size_t)w * 4);
    *words = w;
    return EXCL_OK;
}

extern "C" int excl_parapfd_decode(const uint32_t *in, size_t nwords, uint32_t n, uint32_t *out, size_t *consumed) {
    if (!in || !out || !consumed || nwords == 0) return EXCL_E_INVALID;
    const uint32_t need = pfd_block_words(in, n);
    if (need > nwords) return EXCL_E_FORMAT;
    *consumed = pfd_decode_block(in, n, out);
    return EXCL_OK;
}

extern "C" int excl_newpfd_encode(const uint32_t *in, uint32_t n, float frac, uint32_t *out, size_t cap,
                                  size_t *words) {
    if ((!in && n) || !out || !words) return EXCL_E_INVALID;
    std::vector<uint32_t> tmp((size_t)n * 3 + 8);
    int err = 0;
    const uint32_t w = newpfd_encode_block(in, n, frac, tmp.data(), &err);
    if (err) return err;
    if (w > cap) return EXCL_E_CAPACITY;
    std::memcpy(out, tmp.data(), (size_t)w * 4);
    *words = w;
    return EXCL_OK;
}

extern "C" int excl_newpfd_decode(const uint32_t *in, size_t nwords, uint32_t n, uint32_t *out, size_t *consumed) {
    if (!in || !out || !consumed || nwords == 0) return EXCL_E_INVALID;
    if (newpfd_block_words(in, n, nwords) > nwords) return EXCL_E_FORMAT;
    *consumed = newpfd_decode_block(in, n, out);
    return EXCL_OK;
}

static float g_frac = 0.0f;
extern "C" void excl_set_frac(float frac) { g_frac = frac; }

extern "C" uint32_t encodeArray(const uint32_t *in, uint32_t *out, uint32_t n) {
    int err = 0;
    std::vector<uint32_t> tmp((size_t)n * 3 + 8);
    const uint32_t w = pfd_encode_block(in, n, g_frac, tmp.data(), &err);
    if (err) return 0;
    std::memcpy(out, tmp.data(), (size_t)w * 4);
    return w;
}

extern "C" uint32_t decodeArray(const uint32_t *in, uint32_t *out, uint32_t n) { return pfd_decode_block(in, n, out); }

// ---------------------------------------------------------------------------
// Index build / export.

extern "C" int excl_index_build(const uint32_t *docs, const uint64_t *list_offsets, uint32_t nlists,
                                const excl_build_params *params, excl_index **out) {
    if (!params || !out) return EXCL_E_INVALID;
    excl_index *ix = new (std::nothrow) excl_index();
    if (!ix) return EXCL_E_NOMEM;
    std::string err;
    int st;
    try {
        st = build_index(docs, list_offsets, nlists, *params, *ix, err);
    } catch (const std::bad_alloc &) {
        st = EXCL_E_NOMEM;
    }
    if (st) {
        std::fprintf(stderr, "excl_index_build: %s\n", err.c_str());
        delete ix;
        return st;
    }
    *out = ix;
    return EXCL_OK;
}

extern "C" int excl_index_sizes_get(const excl_index *ix, excl_index_sizes *s) {
    if (!ix || !s) return EXCL_E_INVALID;
    s->nlists = ix->nlists;
    s->nsegs = ix->seg_head.size();
    s->nwords = ix->words.size();
    s->ndir = ix->dir.size();
    s->ntilemap = ix->tilemap.size();
    s->postings = ix->postings;
    s->device_bytes = ix->dev ? ix->dev->bytes : 0;
    return EXCL_OK;
}

extern "C" int excl_index_export(const excl_index *ix, excl_list_info *lists, uint32_t *words, uint32_t *seg_head,
                                 uint32_t *seg_rec, uint32_t *seg_reg, uint32_t *dir) {
    if (!ix) return EXCL_E_INVALID;
    if (lists)
        for (uint32_t l = 0; l < ix->nlists; ++l) {
            const ListDesc &d = ix->lists[l];
            excl_list_info &o = lists[l];
            o.word_base = d.word_base;
            o.n = d.n;
            o.seg_base = d.seg_base;
            o.nseg = d.nseg;
            o.codec = d.codec;
            o.log2_block = d.log2_block;
            o.first_doc = d.first_doc;
            o.last_doc = d.last_doc;
            std::memcpy(o.reg, d.reg, sizeof(o.reg));
            o.dir_shift = d.dir_shift;
            o.dir_base = d.dir_base;
            o.ndir = d.ndir;
            o.tile_base = d.tile_base;
            o.ntiles = d.ntiles;
            o.model = d.model;
        }
    if (words) std::memcpy(words, ix->words.data(), ix->words.size() * 4);
    if (seg_head) std::memcpy(seg_head, ix->seg_head.data(), ix->seg_head.size() * 4);
    if (seg_rec) std::memcpy(seg_rec, ix->seg_rec.data(), ix->seg_rec.size() * sizeof(SegRec));
    if (seg_reg) std::memcpy(seg_reg, ix->seg_reg.data(), ix->seg_reg.size() * sizeof(SegReg));
    if (dir) std::memcpy(dir, ix->dir.data(), ix->dir.size() * 4);
    return EXCL_OK;
}

// ---------------------------------------------------------------------------
// Context.

namespace excl {

void ctx_error(excl_ctx *ctx, const char *fmt, ...) {
    if (!ctx) return;
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->last_error = buf;
}

int cuda_status(excl_ctx *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return EXCL_OK;
    ctx_error(ctx, "%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? EXCL_E_NOMEM : EXCL_E_CUDA;
}

template <typename T>
static int dalloc(excl_ctx *ctx, T **p, size_t count, const char *what) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cuda_status(ctx, cudaMalloc((void **)p, count * sizeof(T)), what);
}

void DeviceIndex::release() {
    cudaFree(lists);
    cudaFree(words);
    cudaFree(seg_head);
    cudaFree(seg_rec);
    cudaFree(seg_reg);
    cudaFree(dir);
    cudaFree(tilemap);
    cudaFree(post_base);
    cudaFree(seg_list);
    cudaFree(seg_gword);
    cudaFree(seg_probe);
    seg_list = nullptr;
    seg_gword = nullptr;
    seg_probe = nullptr;
    lists = nullptr;
    words = seg_head = dir = nullptr;
    seg_rec = nullptr;
    seg_reg = nullptr;
    tilemap = post_base = nullptr;
}

DevIndexView DeviceIndex::view(const ModelView &mv) const {
    DevIndexView v{};
    v.lists = lists;
    v.words = words;
    v.seg_head = seg_head;
    v.seg_rec = seg_rec;
    v.seg_reg = seg_reg;
    v.dir = dir;
    v.tilemap = tilemap;
    v.post_base = post_base;
    v.seg_list = seg_list;
    v.seg_gword = seg_gword;
    v.seg_probe = seg_probe;
    v.models = mv;
    v.codec_mask = codec_mask;
    return v;
}

int ctx_alloc_batch(excl_ctx *ctx) {
    const excl_ctx_config &c = ctx->cfg;
    // Tiles hold >= kMinBlock keys except where consecutive HS segments are
    // grouped (two neighbouring tiles always hold > 256 keys) or a list ends,
    // so this bounds them; larger batches raise EXCL_E_CAPACITY.
    ctx->max_tiles = (uint32_t)std::min<uint64_t>(0xfffffff0ull, c.max_keys / kMinBlock + c.max_queries + 1);
    int st = 0;
    st |= dalloc(ctx, &ctx->d_terms, (size_t)c.max_queries * kMaxTerms, "alloc terms");
    st |= dalloc(ctx, &ctx->d_toff, (size_t)c.max_queries + 1, "alloc term offsets");
    st |= dalloc(ctx, &ctx->d_qterms, (size_t)c.max_queries * kMaxTerms, "alloc qterms");
    st |= dalloc(ctx, &ctx->d_qnterms, (size_t)c.max_queries, "alloc qnterms");
    st |= dalloc(ctx, &ctx->d_tile_prefix, (size_t)c.max_queries + 2, "alloc tile prefix");
    st |= dalloc(ctx, &ctx->d_key_base, (size_t)c.max_queries + 2, "alloc key base");
    st |= dalloc(ctx, &ctx->d_tile_q, (size_t)ctx->max_tiles + 1, "alloc tile owner");
    st |= dalloc(ctx, &ctx->d_tile_count, (size_t)ctx->max_tiles + 1, "alloc tile count");
    st |= dalloc(ctx, &ctx->d_tile_slot, (size_t)ctx->max_tiles + 1, "alloc tile slot");
    st |= dalloc(ctx, &ctx->d_tile_order, (size_t)ctx->max_tiles + 1, "alloc tile order");
    st |= dalloc(ctx, &ctx->d_scratch, (size_t)c.max_keys, "alloc scratch");
    st |= dalloc(ctx, &ctx->d_misc, kMiscWords, "alloc misc");
    st |= dalloc(ctx, &ctx->d_stats, 8, "alloc stats");
    st |= dalloc(ctx, &ctx->d_sync, 1, "alloc pack sync");
    st |= dalloc(ctx, &ctx->d_chunk_state, (size_t)ctx->max_tiles / kSSChunk + 2, "alloc chunk states");
    st |= dalloc(ctx, &ctx->d_offsets, (size_t)c.max_queries + 1, "alloc offsets");
    ctx->docids_cap = c.max_keys;
    st |= dalloc(ctx, &ctx->d_docids, ctx->docids_cap, "alloc docids");
    st |= cuda_status(ctx, cudaMallocHost((void **)&ctx->h_terms, (size_t)c.max_queries * kMaxTerms * 4), "pinned");
    st |= cuda_status(ctx, cudaMallocHost((void **)&ctx->h_toff, ((size_t)c.max_queries + 1) * 4), "pinned");
    st |= cuda_status(ctx, cudaMallocHost((void **)&ctx->h_offsets, ((size_t)c.max_queries + 1) * 4), "pinned");
    st |= cuda_status(ctx, cudaHostAlloc((void **)&ctx->h_flags, kFlagSlots * 4, cudaHostAllocMapped), "pinned");
    if (!st) st |= cuda_status(ctx, cudaHostGetDevicePointer((void **)&ctx->m_flags, ctx->h_flags, 0), "mapped flags");
    if (st) return EXCL_E_NOMEM;
    for (uint32_t i = kFlagSlots; i-- > 0;) ctx->free_flag_slots.push_back(i);
    cudaMemsetAsync(ctx->d_misc, 0, kMiscWords * 4, ctx->stream);
    cudaMemsetAsync(ctx->d_stats, 0, 8 * 8, ctx->stream);
    cudaMemsetAsync(ctx->d_sync, 0, sizeof(PackSync), ctx->stream);
    cudaMemsetAsync(ctx->d_chunk_state, 0, ((size_t)ctx->max_tiles / kSSChunk + 2) * 8, ctx->stream);
    return cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "ctx init");
}

uint32_t host_batch_tiles(const excl_ctx *ctx, const excl_index *ix, const uint32_t *terms,
                          const uint32_t *term_offsets, uint32_t nq) {
    if (nq > kHostTilesMaxQueries || !terms) return 0;
    uint64_t tiles = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        const ListDesc *best = nullptr;
        for (uint32_t i = term_offsets[q]; i < term_offsets[q + 1]; ++i) {
            const uint32_t t = terms[i];
            if (t < ix->nlists && (!best || ix->lists[t].n < best->n)) best = &ix->lists[t];
        }
        if (best) tiles += split_tiles(best->n, best->ntiles, best->log2_block, ctx->tile_split);
    }
    return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(tiles, 1), 0xffffffffu);
}

// Runs the whole device pipeline for nq queries whose terms are in device memory.
int run_pipeline(excl_ctx *ctx, excl_index *ix, const uint32_t *d_terms, const uint32_t *d_toff, uint32_t nq,
                 uint32_t algo, uint32_t *d_offsets, uint32_t *d_docids, uint64_t cap, uint32_t *err_out,
                 uint32_t tiles_hint) {
    if (!ix->dev) {
        ctx_error(ctx, "index not uploaded");
        return EXCL_E_INVALID;
    }
    if (nq > ctx->cfg.max_queries) {
        ctx_error(ctx, "batch of %u queries exceeds max_queries %u", nq, ctx->cfg.max_queries);
        return EXCL_E_CAPACITY;
    }
    if (algo > EXCL_ALGO_SEGREG) {
        ctx_error(ctx, "unknown algo %u", algo);
        return EXCL_E_INVALID;
    }
    if (algo == EXCL_ALGO_AUTO && ctx->tuned_algo >= 0) algo = (uint32_t)ctx->tuned_algo;
    cudaStream_t st = ctx->stream;
    BatchView b{};
    b.nq = nq;
    b.qterms = ctx->d_qterms;
    b.qnterms = ctx->d_qnterms;
    b.tile_prefix = ctx->d_tile_prefix;
    b.tile_q = ctx->d_tile_q;
    b.tile_counter = ctx->d_misc + kMiscTileCounter;
    b.key_base = ctx->d_key_base;
    b.tile_count = ctx->d_tile_count;
    b.tile_slot = ctx->d_tile_slot;
    b.tile_order = ctx->d_tile_order;
    b.scratch = ctx->d_scratch;
    b.max_tiles = ctx->max_tiles;
    b.merge_segs = ctx->merge_segs;
    b.tile_split = ctx->tile_split;
    b.max_keys = ctx->cfg.max_keys;
    b.err = ctx->d_misc + kMiscErr;
    b.err_out = err_out;
    b.probe_done = ctx->d_misc + kMiscProbeDone;
    b.scatter_ready = ctx->d_misc + kMiscScatterReady;
    b.check_polls = ctx->wait_check_polls;
    b.check_flag = ctx->d_misc + kMiscNeverSet;
    b.stats = ctx->collect_stats ? ctx->d_stats : nullptr;
    BatchLaunch L{};
    L.ixv = ix->dev->view(ix->models ? model_view(ix->models) : ModelView{});
    L.lists = ix->dev->lists;
    L.nlists = ix->nlists;
    L.terms = d_terms;
    L.toff = d_toff;
    L.b = b;
    L.sync = ctx->d_sync;
    L.chunk_state = ctx->d_chunk_state;
    L.offsets = d_offsets;
    L.docids = d_docids;
    L.cap = cap;
    L.algo = (int)algo;
    L.warps = ctx->warps;
    L.ctas_per_sm = ctx->ctas_per_sm;
    L.nsm = ctx->nsm;
    L.max_ctas = tiles_hint ? std::max<uint32_t>(1, (tiles_hint + kBatchWarps - 1) / kBatchWarps) : 0u;
    L.spin = ctx->spin_limit;
    L.ev = ctx->ev;
    ctx->last_was_graph = false;
    if (ctx->use_graphs) {
        // the key covers every launch argument: the device view of the index
        // (hashed, so a re-upload or new models recapture) and the batch's buffers
        uint64_t vh = 1469598103934665603ull;
        const unsigned char *vb = reinterpret_cast<const unsigned char *>(&L.ixv);
        for (size_t i = 0; i < sizeof L.ixv; ++i) vh = (vh ^ vb[i]) * 1099511628211ull;
        const uint64_t key[12] = {(uint64_t)(uintptr_t)ix, vh, (uint64_t)(uintptr_t)d_terms,
                                  (uint64_t)(uintptr_t)d_toff, nq, algo, (uint64_t)(uintptr_t)d_offsets,
                                  (uint64_t)(uintptr_t)d_docids, cap,
                                  (uint64_t)ctx->collect_stats | (uint64_t)ctx->merge_segs << 8 |
                                      (uint64_t)ctx->warps << 16 | (uint64_t)ctx->ctas_per_sm << 32 |
                                      (uint64_t)ctx->tile_split << 40 | (uint64_t)(ctx->spin_limit != 0) << 48 |
                                      (uint64_t)(ctx->wait_check_polls != 0) << 49,
                                  (uint64_t)(uintptr_t)err_out, L.max_ctas};
        const bool same = ctx->gkey_seen && std::memcmp(key, ctx->gkey, sizeof key) == 0;
        if (same || ctx->gexec) {
            if (!same || !ctx->gexec) {
                // capture this argument set once and update the executable graph in place
                L.ev = nullptr;
                cudaGraph_t g = nullptr;
                int e = cuda_status(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
                if (!e) {
                    const int le = launch_batch(L, st);
                    e = cuda_status(ctx, cudaStreamEndCapture(st, &g), "end capture");
                    if (!e && le) e = cuda_status(ctx, (cudaError_t)le, "launch in capture");
                }
                if (!e && ctx->gexec) {
                    cudaGraphExecUpdateResultInfo info;
                    if (cudaGraphExecUpdate(ctx->gexec, g, &info) != cudaSuccess) {
                        cudaGetLastError();
                        cudaGraphExecDestroy(ctx->gexec);
                        ctx->gexec = nullptr;
                    }
                }
                if (!e && !ctx->gexec) e = cuda_status(ctx, cudaGraphInstantiate(&ctx->gexec, g, 0), "instantiate");
                if (g) cudaGraphDestroy(g);
                if (e) return e;
                std::memcpy(ctx->gkey, key, sizeof key);
                ctx->gkey_seen = true;
            }
            cudaEventRecord(ctx->ev[0], st);
            const int e = cuda_status(ctx, cudaGraphLaunch(ctx->gexec, st), "graph launch");
            cudaEventRecord(ctx->ev[3], st);
            if (e) return e;
            ctx->last_was_graph = true;
            ctx->last_nq = nq;
            return EXCL_OK;
        }
        // first sighting of this argument set: run it uncaptured
        std::memcpy(ctx->gkey, key, sizeof key);
        ctx->gkey_seen = true;
    }
    const int e = launch_batch(L, st);
    if (e) return cuda_status(ctx, (cudaError_t)e, "launch");
    ctx->last_nq = nq;
    return EXCL_OK;
}

int read_device_flags(excl_ctx *ctx) {
    uint32_t f = 0;
    cudaError_t e = cudaMemcpy(&f, ctx->d_misc + kMiscErr, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(ctx, e, "read error flag");
    if (f) cudaMemset(ctx->d_misc + kMiscErr, 0, 4);
    return flags_status(ctx, f);
}

// Maps a batch's device error word to a status (and the context's message).
int flags_status(excl_ctx *ctx, uint32_t f) {
    if (f) {
        ctx_error(ctx, "device error flags 0x%x (%s%s%s%s%s)", f, (f & kErrTerms) ? "too many terms " : "",
                  (f & kErrScanSpin) ? "scan wait expired " : "", (f & kErrTermId) ? "term id out of range " : "",
                  (f & kErrCapacity) ? "result capacity " : "", (f & kErrModel) ? "model " : "");
        if (f & kErrCapacity) return EXCL_E_CAPACITY;
        if (f & (kErrTermId | kErrTerms)) return EXCL_E_INVALID;
        return EXCL_E_DEVICE_FLAG;
    }
    return EXCL_OK;
}

}  // namespace excl

extern "C" int excl_ctx_create(int device, const excl_ctx_config *cfg, excl_ctx **out) {
    if (!out) return EXCL_E_INVALID;
    *out = nullptr;
    excl_ctx *ctx = new (std::nothrow) excl_ctx();
    if (!ctx) return EXCL_E_NOMEM;
    ctx->device = device;
    excl_ctx_config c{};
    if (cfg) c = *cfg;
    if (c.max_queries == 0) c.max_queries = 65536;
    if (c.max_queries > kPackMaxQueries) c.max_queries = kPackMaxQueries;
    if (c.max_terms == 0 || c.max_terms > kMaxTerms) c.max_terms = kMaxTerms;
    if (c.max_keys == 0) c.max_keys = 1ull << 26;
    ctx->cfg = c;
    ctx->warps = c.warps_per_cta ? (int)c.warps_per_cta : 8;
    ctx->ctas_per_sm = c.ctas_per_sm ? (int)c.ctas_per_sm : 5;
    ctx->use_graphs = c.use_graphs != 0;
    ctx->merge_segs = c.merge_segs == 0 ? 2u : c.merge_segs == EXCL_MERGE_OFF ? 0u : std::min(c.merge_segs, 4u);
    int st = cuda_status(ctx, cudaSetDevice(device), "cudaSetDevice");
    if (!st) st = cuda_status(ctx, cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device), "attr");
    if (!st) st = cuda_status(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
    for (int i = 0; i < 4 && !st; ++i) st = cuda_status(ctx, cudaEventCreate(&ctx->ev[i]), "event");
    if (!st) st = ctx_alloc_batch(ctx);
    if (st) {
        std::fprintf(stderr, "excl_ctx_create: %s\n", ctx->last_error.c_str());
        excl_ctx_destroy(ctx);
        return st;
    }
    *out = ctx;
    return EXCL_OK;
}

extern "C" int excl_ctx_destroy(excl_ctx *ctx) {
    if (!ctx) return EXCL_E_INVALID;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    uint32_t *bufs[] = {ctx->d_terms,   ctx->d_toff, ctx->d_qterms,   ctx->d_qnterms,   ctx->d_tile_prefix,
                        ctx->d_tile_q,  ctx->d_tile_count, ctx->d_scratch, ctx->d_misc, ctx->d_key_base,
                        ctx->d_tile_slot, reinterpret_cast<uint32_t *>(ctx->d_tile_order), ctx->d_offsets,
                        ctx->d_docids};
    for (uint32_t *p : bufs) cudaFree(p);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    cudaFree(ctx->d_stats);
    cudaFree(ctx->d_sync);
    cudaFree(ctx->d_chunk_state);
    cudaFreeHost(ctx->h_terms);
    cudaFreeHost(ctx->h_toff);
    cudaFreeHost(ctx->h_offsets);
    cudaFreeHost(ctx->h_flags);
    for (cudaEvent_t &e : ctx->slot_ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return EXCL_OK;
}

extern "C" const char *excl_last_error(const excl_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

extern "C" void *excl_ctx_stream(excl_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" int excl_index_upload(excl_ctx *ctx, excl_index *ix) {
    if (!ctx || !ix) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    cudaSetDevice(ctx->device);
    if (ix->dev) {
        ix->dev->release();
        delete ix->dev;
        ix->dev = nullptr;
    }
    DeviceIndex *d = new (std::nothrow) DeviceIndex();
    if (!d) return EXCL_E_NOMEM;
    std::vector<uint64_t> pb(ix->nlists + 1, 0);
    for (uint32_t l = 0; l < ix->nlists; ++l) pb[l + 1] = pb[l] + ix->lists[l].n;
    // per-segment list id and global block start (blocks of consecutive
    // segments are contiguous, so a block ends where the next one starts)
    const size_t nsegs = ix->seg_head.size();
    std::vector<uint32_t> slist(nsegs);
    std::vector<uint64_t> sgw(nsegs + 1);
    for (uint32_t l = 0; l < ix->nlists; ++l)
        for (uint32_t s = 0; s < ix->lists[l].nseg; ++s) {
            const size_t g = (size_t)ix->lists[l].seg_base + s;
            slist[g] = l;
            sgw[g] = ix->lists[l].word_base + ix->seg_rec[g].off;
        }
    sgw[nsegs] = ix->words.size() - kWordPad;
    std::vector<ProbeRec> prec(nsegs);
    for (size_t g = 0; g < nsegs; ++g) {
        const SegRec &r = ix->seg_rec[g];
        const SegReg &rg = ix->seg_reg[g];
        ProbeRec &p = prec[g];
        std::memset(&p, 0, sizeof p);
        p.head = ix->seg_head[g];
        p.off = r.off;
        p.aux = r.aux;
        p.count = r.count;
        p.hdr = ix->words[sgw[g]];
        p.a = rg.a;
        p.b = rg.b;
        p.lr = std::min<uint32_t>(rg.L, kProbeUnbounded) | std::min<uint32_t>(rg.R, kProbeUnbounded) << 16;
        p.start = r.start;
        const ListDesc &L = ix->lists[slist[g]];
        p.codec = L.codec;
        p.ob = pb[slist[g]] + r.start;
        p.r0 = L.reg[0];
        p.r1 = L.reg[1];
    }
    int st = 0;
    st |= dalloc(ctx, &d->lists, ix->lists.size(), "index lists");
    st |= dalloc(ctx, &d->words, ix->words.size(), "index words");
    st |= dalloc(ctx, &d->seg_head, ix->seg_head.size(), "index heads");
    st |= dalloc(ctx, &d->seg_rec, ix->seg_rec.size(), "index recs");
    st |= dalloc(ctx, &d->seg_reg, ix->seg_reg.size(), "index regs");
    st |= dalloc(ctx, &d->dir, ix->dir.size(), "index dir");
    st |= dalloc(ctx, &d->tilemap, ix->tilemap.size(), "index tilemap");
    st |= dalloc(ctx, &d->post_base, pb.size(), "index post base");
    st |= dalloc(ctx, &d->seg_list, slist.size(), "index seg list");
    st |= dalloc(ctx, &d->seg_gword, sgw.size(), "index seg words");
    st |= dalloc(ctx, &d->seg_probe, prec.size(), "index probe records");
    if (st) {
        d->release();
        delete d;
        return EXCL_E_NOMEM;
    }
    auto up = [&](void *dst, const void *src, size_t bytes) {
        if (bytes && !st) st = cuda_status(ctx, cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), "index upload");
    };
    up(d->lists, ix->lists.data(), ix->lists.size() * sizeof(ListDesc));
    up(d->words, ix->words.data(), ix->words.size() * 4);
    up(d->seg_head, ix->seg_head.data(), ix->seg_head.size() * 4);
    up(d->seg_rec, ix->seg_rec.data(), ix->seg_rec.size() * sizeof(SegRec));
    up(d->seg_reg, ix->seg_reg.data(), ix->seg_reg.size() * sizeof(SegReg));
    up(d->dir, ix->dir.data(), ix->dir.size() * 4);
    up(d->tilemap, ix->tilemap.data(), ix->tilemap.size() * 8);
    up(d->post_base, pb.data(), pb.size() * 8);
    up(d->seg_list, slist.data(), slist.size() * 4);
    up(d->seg_gword, sgw.data(), sgw.size() * 8);
    up(d->seg_probe, prec.data(), prec.size() * sizeof(ProbeRec));
    if (st) {
        d->release();
        delete d;
        return st;
    }
    d->bytes = ix->lists.size() * sizeof(ListDesc) + ix->words.size() * 4 + ix->seg_head.size() * 4 +
               ix->seg_rec.size() * sizeof(SegRec) + ix->seg_reg.size() * sizeof(SegReg) + ix->dir.size() * 4 +
               ix->tilemap.size() * 8 + pb.size() * 8 + slist.size() * 4 + sgw.size() * 8 +
               prec.size() * sizeof(ProbeRec);
    d->device = ctx->device;
    for (uint32_t l = 0; l < ix->nlists; ++l) d->codec_mask |= 1u << ix->lists[l].codec;
    ix->dev = d;
    if (ix->models) st = models_upload(ctx, ix);
    return st;
}

extern "C" int excl_index_free(excl_index *ix) {
    if (!ix) return EXCL_E_INVALID;
    if (ix->dev) {
        cudaSetDevice(ix->dev->device);
        ix->dev->release();
        delete ix->dev;
    }
    if (ix->models) models_free(ix->models);
    delete ix;
    return EXCL_OK;
}

extern "C" int excl_decode_lists_device(excl_ctx *ctx, excl_index *ix, uint32_t l0, uint32_t l1, uint32_t *d_out) {
    if (!ctx || !ix || !d_out || l0 >= l1 || l1 > ix->nlists) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    if (!ix->dev) {
        ctx_error(ctx, "index not uploaded");
        return EXCL_E_INVALID;
    }
    cudaSetDevice(ctx->device);
    uint64_t base0 = 0;
    for (uint32_t l = 0; l < l0; ++l) base0 += ix->lists[l].n;
    const uint32_t seg0 = ix->lists[l0].seg_base;
    const uint32_t seg1 = ix->lists[l1 - 1].seg_base + ix->lists[l1 - 1].nseg;
    const int e = launch_decode(ix->dev->view(ModelView{}), l0, l1, base0, d_out, seg0, seg1 - seg0, ctx->nsm,
                                ctx->d_misc + kMiscDecodeTicket, ctx->d_misc + kMiscErr, ctx->stream);
    return cuda_status(ctx, (cudaError_t)e, "decode launch");
}

extern "C" int excl_decode_lists(excl_ctx *ctx, excl_index *ix, uint32_t l0, uint32_t l1, uint32_t *out, size_t cap) {
    if (!ctx || !ix || !out || l0 >= l1 || l1 > ix->nlists) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    uint64_t n = 0;
    for (uint32_t l = l0; l < l1; ++l) n += ix->lists[l].n;
    if (n > cap) return EXCL_E_CAPACITY;
    cudaSetDevice(ctx->device);
    uint32_t *d = nullptr;
    int st = dalloc(ctx, &d, n, "decode buffer");
    if (st) return st;
    st = excl_decode_lists_device(ctx, ix, l0, l1, d);
    if (!st) st = cuda_status(ctx, cudaMemcpyAsync(out, d, n * 4, cudaMemcpyDeviceToHost, ctx->stream), "decode d2h");
    if (!st) st = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "decode sync");
    cudaFree(d);
    return st;
}

// ---------------------------------------------------------------------------
// Batches.

extern "C" int excl_intersect_device(excl_ctx *ctx, excl_index *ix, const uint32_t *d_terms,
                                     const uint32_t *d_term_offsets, uint32_t nq, uint32_t algo, uint32_t *d_offsets,
                                     uint32_t *d_docids, uint64_t cap) {
    if (!ctx || !ix || !d_term_offsets || !d_offsets || (!d_docids && cap)) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    cudaSetDevice(ctx->device);
    return run_pipeline(ctx, ix, d_terms, d_term_offsets, nq, algo, d_offsets, d_docids, cap);
}

extern "C" int excl_ctx_check(excl_ctx *ctx) {
    if (!ctx) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    cudaSetDevice(ctx->device);
    int st = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "stream sync");
    if (st) return st;
    return read_device_flags(ctx);
}

struct excl_batch {
    excl_ctx *ctx;
    uint32_t nq;
    cudaEvent_t done;  // the slot's event (owned by the context)
    bool waited;
    const uint32_t *into_offsets = nullptr;  // excl_submit_into: the caller's offsets array
    int32_t slot = -1;                       // this batch's slot: error word in ctx->h_flags, event
    uint64_t seq = 0;                        // excl_submit: its number among the context's excl_submit batches
};

// A free batch slot (its pinned error word cleared), or -1 with the context's
// error set. The caller holds ctx->op_mu.
static int32_t take_slot(excl_ctx *ctx) {
    using namespace excl;
    if (ctx->free_flag_slots.empty()) {
        ctx_error(ctx, "more than %u batches in flight", kFlagSlots);
        return -1;
    }
    const uint32_t slot = ctx->free_flag_slots.back();
    if (!ctx->slot_ev[slot] && cudaEventCreateWithFlags(&ctx->slot_ev[slot], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        ctx->slot_ev[slot] = nullptr;
        ctx_error(ctx, "event");
        return -1;
    }
    ctx->free_flag_slots.pop_back();
    ctx->h_flags[slot] = 0;
    return (int32_t)slot;
}

// Ends a batch whose pipeline ran with err_out = the slot's mapped word (the
// batch kernel's last CTA hands the batch's error bits to it and clears the device
// word, so batches in flight together each see their own flags): records the
// slot's event and hands the batch out. On failure the slot is returned.
static int finish_batch(excl_ctx *ctx, uint32_t nq, int32_t slot, const uint32_t *into_offsets, excl_batch **ticket) {
    using namespace excl;
    excl_batch *b = new (std::nothrow) excl_batch{ctx, nq, ctx->slot_ev[slot], false};
    int s = b ? cuda_status(ctx, cudaEventRecord(ctx->slot_ev[slot], ctx->stream), "record") : EXCL_E_NOMEM;
    if (s) {
        delete b;
        cudaStreamSynchronize(ctx->stream);  // the batch's kernels may still write the slot
        ctx->free_flag_slots.push_back((uint32_t)slot);
        return s;
    }
    b->slot = slot;
    b->into_offsets = into_offsets;
    *ticket = b;
    return EXCL_OK;
}

// Copies a host batch into the context's query buffers (after the previous
// batch has released them). Returns the number of terms through *nterms.
static int stage_host_batch(excl_ctx *ctx, excl_index *ix, const uint32_t *terms, const uint32_t *term_offsets,
                            uint32_t nq, uint32_t *nterms_out) {
    if (nq > ctx->cfg.max_queries) {
        ctx_error(ctx, "batch of %u queries exceeds max_queries %u", nq, ctx->cfg.max_queries);
        return EXCL_E_CAPACITY;
    }
    const uint32_t nterms = term_offsets[nq] - term_offsets[0];
    if (nterms > (uint64_t)ctx->cfg.max_queries * kMaxTerms) return EXCL_E_CAPACITY;
    for (uint32_t q = 0; q < nq; ++q) {
        if (term_offsets[q + 1] < term_offsets[q]) return EXCL_E_INVALID;
        if (term_offsets[q + 1] - term_offsets[q] > kMaxTerms) {
            ctx_error(ctx, "query %u has more than %u terms", q, kMaxTerms);
            return EXCL_E_CAPACITY;
        }
    }
    for (uint32_t i = 0; i < nterms; ++i)
        if (terms[term_offsets[0] + i] >= ix->nlists) {
            ctx_error(ctx, "term id %u out of range", terms[term_offsets[0] + i]);
            return EXCL_E_INVALID;
        }
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    std::memcpy(ctx->h_terms, terms + term_offsets[0], (size_t)nterms * 4);
    for (uint32_t q = 0; q <= nq; ++q) ctx->h_toff[q] = term_offsets[q] - term_offsets[0];
    int s = cuda_status(ctx, cudaMemcpyAsync(ctx->d_terms, ctx->h_terms, (size_t)nterms * 4, cudaMemcpyHostToDevice,
                                             ctx->stream),
                        "h2d terms");
    if (!s)
        s = cuda_status(ctx, cudaMemcpyAsync(ctx->d_toff, ctx->h_toff, ((size_t)nq + 1) * 4, cudaMemcpyHostToDevice,
                                             ctx->stream),
                        "h2d offsets");
    if (nterms_out) *nterms_out = nterms;
    return s;
}

extern "C" int excl_autotune(excl_ctx *ctx, excl_index *ix, const uint32_t *terms, const uint32_t *term_offsets,
                             uint32_t nq, excl_tune_report *rep) {
    if (!ctx || !ix || !term_offsets || !rep) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    if (!ix->dev) return EXCL_E_INVALID;
    int s = stage_host_batch(ctx, ix, terms, term_offsets, nq, nullptr);
    if (s) return s;
    // candidates are timed without graphs, on the context's own buffers
    const bool graphs = ctx->use_graphs;
    const int w0 = ctx->warps, c0 = ctx->ctas_per_sm, t0 = ctx->tuned_algo;
    const uint32_t m0 = ctx->merge_segs, sp0 = ctx->tile_split;
    ctx->use_graphs = false;
    ctx->tuned_algo = -1;
    ctx->tile_split = 0;
    auto time_one = [&](uint32_t algo, int warps, int ctas, uint32_t merge, float *ms) -> int {
        ctx->warps = warps;
        ctx->ctas_per_sm = ctas;
        ctx->merge_segs = merge;
        float t[3];
        for (int r = 0; r < 4; ++r) {
            int e = run_pipeline(ctx, ix, ctx->d_terms, ctx->d_toff, nq, algo, ctx->d_offsets, ctx->d_docids,
                                 ctx->docids_cap);
            if (!e) e = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "tune sync");
            if (!e) e = read_device_flags(ctx);
            if (e) return e;
            if (r) cudaEventElapsedTime(&t[r - 1], ctx->ev[0], ctx->ev[3]);
        }
        std::sort(t, t + 3);
        *ms = t[1];
        return EXCL_OK;
    };
    std::memset(rep, 0, sizeof *rep);
    s = time_one(EXCL_ALGO_AUTO, 8, 5, 2, &rep->default_ms);
    float best = rep->default_ms;
    uint32_t ba = EXCL_ALGO_AUTO, bm = 2;
    int bw = 8, bc = 5;
    const uint32_t algos[4] = {EXCL_ALGO_BSEARCH, EXCL_ALGO_HASHSEG, EXCL_ALGO_SEGREG, EXCL_ALGO_LEARNED};
    const int warps[1] = {8}, ctas[3] = {4, 5, 6};
    const uint32_t merges[4] = {0u, 1u, 2u, 4u};
    uint32_t tried = 1;
    for (uint32_t a : algos) {
        if (s) break;
        if (a == EXCL_ALGO_LEARNED && !ix->models) continue;
        for (int wv : warps)
            for (int cv : ctas)
                for (uint32_t mv : merges) {
                    if (s) break;
                    float ms = 0;
                    s = time_one(a, wv, cv, mv, &ms);
                    ++tried;
                    if (!s && ms < best) {
                        best = ms;
                        ba = a;
                        bw = wv;
                        bc = cv;
                        bm = mv;
                    }
                }
    }
    // then, with the best setting, fixed segments cut into 2 or 4 tiles
    // (shorter work items: the persistent queue's tail evens out)
    uint32_t bsp = 0;
    for (uint32_t sp = 1; sp <= 2 && !s; ++sp) {
        ctx->tile_split = sp;
        float ms = 0;
        s = time_one(ba, bw, bc, bm, &ms);
        ++tried;
        if (!s && ms < best) {
            best = ms;
            bsp = sp;
        }
    }
    ctx->use_graphs = graphs;
    if (s) {
        ctx->warps = w0;
        ctx->ctas_per_sm = c0;
        ctx->merge_segs = m0;
        ctx->tuned_algo = t0;
        ctx->tile_split = sp0;
        return s;
    }
    ctx->warps = bw;
    ctx->ctas_per_sm = bc;
    ctx->merge_segs = bm;
    ctx->tile_split = bsp;
    ctx->tuned_algo = (int)ba;
    rep->algo = ba;
    rep->warps_per_cta = (uint32_t)bw;
    rep->ctas_per_sm = (uint32_t)bc;
    rep->merge_segs = bm ? bm : EXCL_MERGE_OFF;
    rep->best_ms = best;
    rep->tried = tried;
    rep->tile_split = bsp;
    return EXCL_OK;
}

extern "C" int excl_submit(excl_ctx *ctx, excl_index *ix, const uint32_t *terms, const uint32_t *term_offsets,
                           uint32_t nq, uint32_t algo, excl_batch **ticket) {
    if (!ctx || !ix || !term_offsets || !ticket) return EXCL_E_INVALID;
    *ticket = nullptr;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    cudaStream_t st = ctx->stream;
    int s = stage_host_batch(ctx, ix, terms, term_offsets, nq, nullptr);
    if (s) return s;
    const int32_t slot = take_slot(ctx);
    if (slot < 0) return EXCL_E_CAPACITY;
    s = run_pipeline(ctx, ix, ctx->d_terms, ctx->d_toff, nq, algo, ctx->d_offsets, ctx->d_docids, ctx->docids_cap,
                     ctx->m_flags + slot, host_batch_tiles(ctx, ix, terms, term_offsets, nq));
    if (!s)
        s = cuda_status(ctx, cudaMemcpyAsync(ctx->h_offsets, ctx->d_offsets, ((size_t)nq + 1) * 4,
                                             cudaMemcpyDeviceToHost, st),
                        "d2h offsets");
    if (s) {
        cudaStreamSynchronize(st);
        ctx->free_flag_slots.push_back((uint32_t)slot);
        return s;
    }
    s = finish_batch(ctx, nq, slot, nullptr, ticket);
    if (!s) (*ticket)->seq = ++ctx->submit_seq;
    return s;
}

extern "C" int excl_ctx_set_tuning(excl_ctx *ctx, const excl_tune_report *rep) {
    if (!ctx || !rep) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    if (rep->algo > EXCL_ALGO_SEGREG || (rep->warps_per_cta != 4 && rep->warps_per_cta != 8) ||
        rep->ctas_per_sm < 4 || rep->ctas_per_sm > 6 || rep->tile_split > 2 ||
        (rep->merge_segs != EXCL_MERGE_OFF && (rep->merge_segs == 0 || rep->merge_segs > 4)))
        return EXCL_E_INVALID;
    ctx->warps = (int)rep->warps_per_cta;
    ctx->ctas_per_sm = (int)rep->ctas_per_sm;
    ctx->merge_segs = rep->merge_segs == EXCL_MERGE_OFF ? 0u : rep->merge_segs;
    ctx->tuned_algo = rep->algo == EXCL_ALGO_AUTO ? -1 : (int)rep->algo;
    ctx->tile_split = rep->tile_split;
    return EXCL_OK;
}

extern "C" int excl_autotune_layout(excl_ctx *ctx, const uint32_t *d_docs, const uint64_t *list_offsets,
                                    uint32_t nlists, excl_layout_candidate *cands, uint32_t ncands,
                                    const uint32_t *terms, const uint32_t *term_offsets, uint32_t nq, uint32_t *best,
                                    excl_index **out) {
    if (!ctx || !d_docs || !list_offsets || !cands || !ncands || !term_offsets || !best || !out) return EXCL_E_INVALID;
    *out = nullptr;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    excl_index *keep = nullptr;
    uint32_t kb = ncands;
    for (uint32_t i = 0; i < ncands; ++i) {
        excl_layout_candidate &c = cands[i];
        c.best_ms = 0.0f;
        c.device_bytes = 0;
        std::memset(&c.tuning, 0, sizeof c.tuning);
        excl_index *ix = nullptr;
        c.status = excl_index_build_device(ctx, d_docs, list_offsets, nlists, &c.build, &ix);
        if (!c.status) c.status = excl_index_upload(ctx, ix);
        if (!c.status) c.status = excl_autotune(ctx, ix, terms, term_offsets, nq, &c.tuning);
        if (!c.status) {
            excl_index_sizes sz{};
            excl_index_sizes_get(ix, &sz);
            c.device_bytes = sz.device_bytes;
            c.best_ms = c.tuning.best_ms;
        }
        if (!c.status && (kb == ncands || c.best_ms < cands[kb].best_ms)) {
            if (keep) excl_index_free(keep);
            keep = ix;
            kb = i;
        } else if (ix) {
            excl_index_free(ix);
        }
    }
    if (!keep) {
        ctx_error(ctx, "excl_autotune_layout: no candidate layout could be built and timed");
        return EXCL_E_INVALID;
    }
    // the context keeps the chosen layout's launch setting
    const int s = excl_ctx_set_tuning(ctx, &cands[kb].tuning);
    if (s) {
        excl_index_free(keep);
        return s;
    }
    *best = kb;
    *out = keep;
    return EXCL_OK;
}

extern "C" int excl_ctx_set_wait_check(excl_ctx *ctx, uint32_t polls) {
    if (!ctx) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    ctx->wait_check_polls = polls;
    return EXCL_OK;
}

// excl_submit_into: the inputs are copied from the caller's host arrays on the
// context's stream (asynchronously when they are page-locked) and the scatter
// kernel writes offsets and docIDs through the device mapping of the caller's
// page-locked output arrays, so the results cross PCIe while the last kernel
// runs and excl_wait has nothing left to copy.
extern "C" int excl_submit_into(excl_ctx *ctx, excl_index *ix, const uint32_t *terms, const uint32_t *term_offsets,
                                uint32_t nq, uint32_t algo, uint32_t *offsets, uint32_t *docids, uint64_t cap,
                                excl_batch **ticket) {
    if (!ctx || !ix || !term_offsets || !offsets || !ticket || (!docids && cap) || (!terms && term_offsets[nq]))
        return EXCL_E_INVALID;
    *ticket = nullptr;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    if (nq > ctx->cfg.max_queries) {
        ctx_error(ctx, "batch of %u queries exceeds max_queries %u", nq, ctx->cfg.max_queries);
        return EXCL_E_CAPACITY;
    }
    // per-query term counts and term ids are checked on the device (error flags)
    const uint32_t nterms = term_offsets[nq];
    if (term_offsets[0] > nterms) return EXCL_E_INVALID;
    if (nterms > (uint64_t)ctx->cfg.max_queries * kMaxTerms) {
        ctx_error(ctx, "batch of %u terms exceeds the context's %llu", nterms,
                  (unsigned long long)ctx->cfg.max_queries * kMaxTerms);
        return EXCL_E_CAPACITY;
    }
    cudaSetDevice(ctx->device);
    // device addresses of the caller's arrays: the outputs must be
    // page-locked and mapped; page-locked inputs are read in place by the pack
    // kernel, others are copied to the context's buffers first
    uint32_t *mapped[4] = {nullptr, nullptr, nullptr, nullptr};
    const void *host[4] = {offsets, docids, terms, term_offsets};
    for (int i = 0; i < 4; ++i) {
        if (!host[i]) continue;
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, host[i]) == cudaSuccess && a.type == cudaMemoryTypeHost && a.devicePointer)
            mapped[i] = static_cast<uint32_t *>(a.devicePointer);
        else
            cudaGetLastError();
        if (i < 2 && !mapped[i]) {
            ctx_error(ctx, "%s array is not page-locked, device-mapped host memory", i ? "docids" : "offsets");
            return EXCL_E_INVALID;
        }
    }
    cudaStream_t st = ctx->stream;
    int s = EXCL_OK;
    const uint32_t *q_terms = mapped[2], *q_toff = mapped[3];
    if (!q_terms && nterms) {
        s = cuda_status(ctx, cudaMemcpyAsync(ctx->d_terms, terms, (size_t)nterms * 4, cudaMemcpyHostToDevice, st),
                        "h2d terms");
        q_terms = ctx->d_terms;
    }
    if (!q_terms) q_terms = ctx->d_terms;  // no terms: never read
    if (!s && !q_toff) {
        s = cuda_status(ctx, cudaMemcpyAsync(ctx->d_toff, term_offsets, ((size_t)nq + 1) * 4, cudaMemcpyHostToDevice,
                                             st),
                        "h2d term offsets");
        q_toff = ctx->d_toff;
    }
    if (s) return s;
    const int32_t slot = take_slot(ctx);
    if (slot < 0) return EXCL_E_CAPACITY;
    s = run_pipeline(ctx, ix, q_terms, q_toff, nq, algo, mapped[0], mapped[1], cap, ctx->m_flags + slot,
                     host_batch_tiles(ctx, ix, terms, term_offsets, nq));
    if (s) {
        cudaStreamSynchronize(st);
        ctx->free_flag_slots.push_back((uint32_t)slot);
        return s;
    }
    return finish_batch(ctx, nq, slot, offsets, ticket);
}

// Polls the batch's event: spins for the first 2 ms (a batch usually ends
// within tens of microseconds of the call), then sleeps between polls.
static int wait_event(excl_ctx *ctx, cudaEvent_t ev, int timeout_ms) {
    const auto t0 = std::chrono::steady_clock::now();
    for (uint32_t polls = 0;; ++polls) {
        const cudaError_t q = cudaEventQuery(ev);
        if (q == cudaSuccess) return EXCL_OK;
        if (q != cudaErrorNotReady) return cuda_status(ctx, q, "batch");
        if ((polls & 63) == 0 || timeout_ms >= 0) {
            const auto dt = std::chrono::steady_clock::now() - t0;
            if (timeout_ms >= 0 && dt > std::chrono::milliseconds(timeout_ms)) return EXCL_E_TIMEOUT;
            if (dt > std::chrono::milliseconds(2)) std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
}

extern "C" int excl_wait(excl_batch *b, uint32_t *offsets, uint32_t *docids, size_t cap, int timeout_ms,
                         uint64_t *total) {
    if (!b) return EXCL_E_INVALID;
    excl_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    if (b->into_offsets && (offsets || docids)) return EXCL_E_INVALID;
    int s = b->waited ? EXCL_OK : wait_event(ctx, b->done, timeout_ms);
    if (s) return s;
    b->waited = true;
    s = flags_status(ctx, ctx->h_flags[b->slot]);
    if (b->into_offsets) {
        // excl_submit_into batch: the results are already in the caller's arrays
        if (total) *total = b->into_offsets[b->nq];
        return s;
    }
    if (s) return s;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    if (b->seq != ctx->submit_seq) {
        ctx_error(ctx, "a later excl_submit on this context replaced this batch's results");
        return EXCL_E_INVALID;
    }
    const uint32_t tot = ctx->h_offsets[b->nq];
    if (total) *total = tot;
    if (offsets) std::memcpy(offsets, ctx->h_offsets, ((size_t)b->nq + 1) * 4);
    if (docids) {
        if (tot > cap) {
            ctx_error(ctx, "result buffer holds %zu docIDs, batch produced %u", cap, tot);
            return EXCL_E_CAPACITY;
        }
        s = cuda_status(ctx, cudaMemcpyAsync(docids, ctx->d_docids, (size_t)tot * 4, cudaMemcpyDeviceToHost, ctx->stream),
                        "d2h docids");
        if (!s) s = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    }
    b->waited = true;
    return s;
}

extern "C" int excl_host_alloc(size_t bytes, void **out) {
    if (!out) return EXCL_E_INVALID;
    *out = nullptr;
    if (!bytes) return EXCL_OK;
    if (cudaHostAlloc(out, bytes, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return EXCL_E_NOMEM;
    }
    return EXCL_OK;
}

extern "C" int excl_host_free(void *p) {
    if (!p) return EXCL_OK;
    return cudaFreeHost(p) == cudaSuccess ? EXCL_OK : EXCL_E_INVALID;
}

extern "C" int excl_batch_free(excl_batch *b) {
    if (!b) return EXCL_E_INVALID;
    if (b->slot >= 0) {
        // a slot returns to the pool only once its batch's writes have landed
        if (!b->waited) cudaEventSynchronize(b->done);
        std::lock_guard<std::recursive_mutex> g(b->ctx->op_mu);
        b->ctx->free_flag_slots.push_back((uint32_t)b->slot);
    }
    delete b;
    return EXCL_OK;
}

extern "C" int excl_last_stats(excl_ctx *ctx, excl_batch_stats *stt) {
    if (!ctx || !stt) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    cudaSetDevice(ctx->device);
    int s = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (s) return s;
    std::memset(stt, 0, sizeof *stt);
    cudaEventElapsedTime(&stt->total_ms, ctx->ev[0], ctx->ev[3]);
    uint32_t T = 0;
    cudaMemcpy(&T, ctx->d_tile_prefix + ctx->last_nq, 4, cudaMemcpyDeviceToHost);
    stt->tiles = T;
    uint64_t hs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (ctx->collect_stats) cudaMemcpy(hs, ctx->d_stats, sizeof hs, cudaMemcpyDeviceToHost);
    stt->probes = hs[0];
    stt->fallbacks = hs[1];
    stt->keys = hs[2];
    stt->merges = hs[3];
    // phases of the batch kernel from its globaltimer stamps: start, pack
    // phase complete, last warp out of the probe loop, last CTA out
    if (hs[4] && hs[5] >= hs[4] && hs[6] >= hs[5] && hs[7] >= hs[6]) {
        stt->pack_ms = (float)((double)(hs[5] - hs[4]) * 1e-6);
        stt->probe_ms = (float)((double)(hs[6] - hs[5]) * 1e-6);
        stt->compact_ms = (float)((double)(hs[7] - hs[6]) * 1e-6);
    }
    return EXCL_OK;
}

extern "C" int excl_checksum(uint32_t nq, const uint32_t *offsets, const uint32_t *docids, uint64_t cs[3]) {
    if (!offsets || !cs) return EXCL_E_INVALID;
    cs[0] = cs[1] = cs[2] = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t n = offsets[q + 1] - offsets[q];
        if (!n) {
            ++cs[0];
            continue;
        }
        const uint32_t *r = docids + offsets[q];
        cs[1] += n;
        cs[2] ^= r[0];
        cs[2] ^= r[n - 1];
        cs[2] ^= r[n / 2];
    }
    return EXCL_OK;
}
