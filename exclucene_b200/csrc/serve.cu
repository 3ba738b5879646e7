// Serving loop: continuous batching of single conjunctive queries on a
// resident index. It has no counterpart in the reference, whose benchmark
// binaries run fixed-size batches read from a query file
// (ParaPFD_Intersection.cu:406-540).
//
//   submit (any thread)  validates the query, works out its shortest list's
//                        docIDs and tiles, queues it.
//   dispatcher thread    whenever a slot is idle, packs the queue head into
//                        one batch: FIFO, up to max_batch_queries and
//                        max_batch_keys, and only as much as fits in the
//                        largest free block of the device working-set pool
//                        (admission by HBM bytes); copies it to the device and
//                        launches the batch pipeline on the slot's stream.
//   slot threads         one per slot: waits for its batch's event, hands
//                        every query its docIDs, frees the pool block.
//
// A slot is a stream with its own cross-CTA pipeline state, error flag and
// pinned host buffers, so batches of different slots overlap on the GPU while
// new queries keep arriving. The batch kernel writes each batch's offsets
// and docIDs straight into the slot's mapped pinned host buffers, so a result
// needs no copy back after the batch event.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "kernels.h"
#include "runtime.h"

namespace excl {
namespace {

using Clock = std::chrono::steady_clock;

constexpr uint64_t up256(uint64_t b) { return (b + 255) & ~255ull; }

// Byte layout of one batch's block of the pool (the queries themselves stay
// in the slot's mapped host arrays).
struct WsLayout {
    uint64_t qterms, qnterms, tile_prefix, key_base, tile_q, tile_count, tile_slot, tile_order, scratch, total;
};

WsLayout ws_layout(uint64_t nq, uint64_t /*nterms*/, uint64_t tiles, uint64_t keys) {
    WsLayout L{};
    uint64_t o = 0;
    auto take = [&](uint64_t words) {
        const uint64_t r = o;
        o += up256(std::max<uint64_t>(words, 1) * 4);
        return r;
    };
    L.qterms = take(nq * kMaxTerms);
    L.qnterms = take(nq);
    L.tile_prefix = take(nq + 2);
    L.key_base = take(nq + 2);
    L.tile_q = take(tiles + 1);
    L.tile_count = take(tiles + 1);
    L.tile_slot = take(tiles + 1);
    L.tile_order = take(4 * (tiles + 1));
    L.scratch = take(keys);
    L.total = o;
    return L;
}

// First-fit allocator over the device pool (host-side bookkeeping only).
class PoolAlloc {
  public:
    void init(uint64_t size) {
        free_.clear();
        free_[0] = size;
    }
    uint64_t largest() const {
        uint64_t m = 0;
        for (const auto &kv : free_) m = std::max(m, kv.second);
        return m;
    }
    bool alloc(uint64_t bytes, uint64_t *off) {
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= bytes) {
                *off = it->first;
                const uint64_t rest = it->second - bytes, at = it->first + bytes;
                free_.erase(it);
                if (rest) free_[at] = rest;
                return true;
            }
        return false;
    }
    void release(uint64_t off, uint64_t bytes) {
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }

  private:
    std::map<uint64_t, uint64_t> free_;
};

struct Replay {
    double *latency_s = nullptr;
    std::atomic<uint64_t> cs0{0}, cs1{0}, cs2{0};
    std::atomic<uint32_t> remaining{0};
    std::atomic<int> status{EXCL_OK};
};

struct Request {
    uint64_t id = 0;
    std::vector<uint32_t> terms;
    uint32_t keys = 0, tiles = 0;
    Clock::time_point t_submit;
    std::vector<uint32_t> result;
    int status = EXCL_OK;
    bool done = false;
    Replay *replay = nullptr;
    uint32_t replay_q = 0;
};
using ReqPtr = std::shared_ptr<Request>;

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    PackSync *d_sync = nullptr;
    uint64_t *d_chunk = nullptr;
    uint32_t *d_misc = nullptr;                      // error flag, probe work counter, tiles probed
    uint32_t *h_terms = nullptr, *h_toff = nullptr;  // pinned, mapped: the pack phase reads them in place
    uint32_t *h_err = nullptr;                       // pinned, mapped: the batch's error bits, handed over by the batch kernel's last CTA
    uint32_t *m_terms = nullptr, *m_toff = nullptr, *m_err = nullptr;  // their device addresses
    uint32_t *h_offsets = nullptr, *h_docids = nullptr;  // mapped pinned results
    uint32_t *m_offsets = nullptr, *m_docids = nullptr;  // their device addresses
    std::vector<ReqPtr> batch;
    uint64_t pool_off = 0, pool_bytes = 0;
    bool busy = false, has_work = false;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
};

}  // namespace
}  // namespace excl

using namespace excl;

struct excl_server {
    int device = 0;
    int nsm = 148;
    excl_index *ix = nullptr;
    excl_server_config cfg{};
    uint32_t slot_max_tiles = 0;
    uint8_t *d_pool = nullptr;
    uint64_t pool_size = 0;
    PoolAlloc pool;
    std::vector<std::unique_ptr<Slot>> slots;
    std::mutex mu;
    std::condition_variable cv_dispatch, cv_done;
    std::deque<ReqPtr> queue;
    std::unordered_map<uint64_t, ReqPtr> tickets;
    uint64_t next_id = 1;
    bool stop = false, stop_slots = false;
    std::thread dispatcher;
    // statistics
    std::vector<float> lat_us;
    uint64_t submitted = 0, completed = 0, batches = 0, rejected = 0, pool_in_use = 0, pool_peak = 0;
    uint32_t inflight = 0, max_inflight = 0;
    int sticky = EXCL_OK;  // first CUDA failure; the server refuses work after it
};

namespace {

int fail_status(uint32_t flags) {
    if (flags & kErrCapacity) return EXCL_E_CAPACITY;
    if (flags & (kErrTermId | kErrTerms)) return EXCL_E_INVALID;
    return flags ? EXCL_E_DEVICE_FLAG : EXCL_OK;
}

// Called with s->mu held.
void finish_locked(excl_server *s, const ReqPtr &r, int status, Clock::time_point t) {
    r->status = status;
    r->done = true;
    const double lat = std::chrono::duration<double>(t - r->t_submit).count();
    if (r->replay) {
        Replay *rp = r->replay;
        if (rp->latency_s) rp->latency_s[r->replay_q] = lat;
        if (status) rp->status.store(status);
        rp->remaining.fetch_sub(1);
    }
    if (!status) {
        ++s->completed;
        s->lat_us.push_back((float)(lat * 1e6));
    }
}

bool head_can_go(excl_server *s) {
    if (s->queue.empty()) return false;
    bool idle = false;
    for (auto &sl : s->slots) idle |= !sl->busy;
    if (!idle) return false;
    const Request &r = *s->queue.front();
    const uint64_t ws = ws_layout(1, r.terms.size(), r.tiles, r.keys).total;
    if (r.keys > s->cfg.max_batch_keys || r.tiles > s->slot_max_tiles || ws > s->pool_size) return true;  // rejected
    return ws <= s->pool.largest();
}

int launch_on_slot(excl_server *s, Slot *sl, uint64_t nterms, uint64_t tiles, uint64_t keys) {
    const uint32_t nq = (uint32_t)sl->batch.size();
    const WsLayout L = ws_layout(nq, nterms, tiles, keys);
    uint32_t o = 0;
    for (uint32_t i = 0; i < nq; ++i) {
        const Request &r = *sl->batch[i];
        sl->h_toff[i] = o;
        std::memcpy(sl->h_terms + o, r.terms.data(), r.terms.size() * 4);
        o += (uint32_t)r.terms.size();
    }
    sl->h_toff[nq] = o;
    uint8_t *base = s->d_pool + sl->pool_off;
    auto at = [&](uint64_t off) { return reinterpret_cast<uint32_t *>(base + off); };
    cudaStream_t st = sl->stream;
    // no copies: the batch kernel reads the batch's queries from the slot's
    // mapped host arrays, its pack phase resets the tile counters, and its
    // last CTA hands the error bits to h_err and clears the device word for
    // the next batch
    BatchView b{};
    b.nq = nq;
    b.qterms = at(L.qterms);
    b.qnterms = at(L.qnterms);
    b.tile_prefix = at(L.tile_prefix);
    b.tile_q = at(L.tile_q);
    b.tile_counter = sl->d_misc + 1;
    b.key_base = at(L.key_base);
    b.tile_count = at(L.tile_count);
    b.tile_slot = at(L.tile_slot);
    b.tile_order = reinterpret_cast<uint4 *>(at(L.tile_order));
    b.scratch = at(L.scratch);
    b.max_tiles = (uint32_t)tiles;
    b.merge_segs = 2;
    b.max_keys = keys;
    b.err = sl->d_misc;
    b.err_out = sl->m_err;
    b.probe_done = sl->d_misc + 32;  // its own 128-byte line, apart from the queue head
    b.scatter_ready = sl->d_misc + 48;
    b.stats = nullptr;
    BatchLaunch bl{};
    bl.ixv = s->ix->dev->view(s->ix->models ? model_view(s->ix->models) : ModelView{});
    bl.lists = s->ix->dev->lists;
    bl.nlists = s->ix->nlists;
    bl.terms = sl->m_terms;
    bl.toff = sl->m_toff;
    bl.b = b;
    bl.sync = sl->d_sync;
    bl.chunk_state = sl->d_chunk;
    bl.offsets = sl->m_offsets;
    bl.docids = sl->m_docids;
    bl.cap = s->cfg.max_batch_keys;
    bl.algo = (int)s->cfg.algo;
    bl.warps = s->cfg.warps_per_cta ? (int)s->cfg.warps_per_cta : 8;
    bl.ctas_per_sm = s->cfg.ctas_per_sm ? (int)s->cfg.ctas_per_sm : 5;
    bl.nsm = s->nsm;
    // one warp per tile: a batch of a few queries leaves the rest of the
    // device to the batches of the other slots
    bl.max_ctas = (uint32_t)std::max<uint64_t>(1, (tiles + kBatchWarps - 1) / kBatchWarps);
    bl.ev = nullptr;
    if (launch_batch(bl, st)) return EXCL_E_CUDA;
    return cudaEventRecord(sl->done, st) == cudaSuccess ? EXCL_OK : EXCL_E_CUDA;
}

void dispatch_loop(excl_server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_dispatch.wait(lk, [&] { return s->stop || head_can_go(s); });
        if (s->stop) break;
        Slot *sl = nullptr;
        for (auto &x : s->slots)
            if (!x->busy) {
                sl = x.get();
                break;
            }
        // FIFO batch from the queue head, within the slot's and the pool's limits
        const uint64_t largest = s->pool.largest();
        uint64_t nterms = 0, tiles = 0, keys = 0;
        sl->batch.clear();
        while (!s->queue.empty() && sl->batch.size() < s->cfg.max_batch_queries) {
            const ReqPtr &r = s->queue.front();
            const uint64_t ws = ws_layout(sl->batch.size() + 1, nterms + r->terms.size(), tiles + r->tiles,
                                          keys + r->keys).total;
            if (keys + r->keys > s->cfg.max_batch_keys || tiles + r->tiles > s->slot_max_tiles || ws > largest) {
                const uint64_t alone = ws_layout(1, r->terms.size(), r->tiles, r->keys).total;
                if (sl->batch.empty() &&
                    (r->keys > s->cfg.max_batch_keys || r->tiles > s->slot_max_tiles || alone > s->pool_size)) {
                    ++s->rejected;  // can never run: larger than a slot or the whole pool
                    finish_locked(s, r, EXCL_E_CAPACITY, Clock::now());
                    s->queue.pop_front();
                    s->cv_done.notify_all();
                    continue;
                }
                break;
            }
            nterms += r->terms.size();
            tiles += r->tiles;
            keys += r->keys;
            sl->batch.push_back(r);
            s->queue.pop_front();
        }
        if (sl->batch.empty()) continue;
        const uint64_t ws = ws_layout(sl->batch.size(), nterms, tiles, keys).total;
        if (!s->pool.alloc(ws, &sl->pool_off)) {  // cannot happen: ws <= largest free block
            // back to the queue head in their original (FIFO) order
            for (auto it = sl->batch.rbegin(); it != sl->batch.rend(); ++it) s->queue.push_front(*it);
            sl->batch.clear();
            continue;
        }
        sl->pool_bytes = ws;
        sl->busy = true;
        s->pool_in_use += ws;
        s->pool_peak = std::max(s->pool_peak, s->pool_in_use);
        ++s->batches;
        ++s->inflight;
        s->max_inflight = std::max(s->max_inflight, s->inflight);
        const int sticky = s->sticky;
        lk.unlock();
        int st = sticky ? sticky : launch_on_slot(s, sl, nterms, tiles, keys);
        {
            std::lock_guard<std::mutex> g(sl->mu);
            sl->has_work = true;
            if (st) sl->pool_bytes |= 1ull << 63;  // tells the slot thread the launch failed
        }
        sl->cv.notify_one();
        lk.lock();
        if (st && !s->sticky) s->sticky = st;
    }
    // fail what is still queued
    for (auto &r : s->queue) finish_locked(s, r, EXCL_E_INVALID, Clock::now());
    s->queue.clear();
    s->cv_done.notify_all();
}

void slot_loop(excl_server *s, Slot *sl) {
    cudaSetDevice(s->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> g(sl->mu);
            sl->cv.wait(g, [&] { return sl->has_work || s->stop_slots; });
            if (!sl->has_work) break;
        }
        const bool launch_failed = (sl->pool_bytes >> 63) != 0;
        sl->pool_bytes &= ~(1ull << 63);
        int status = launch_failed ? EXCL_E_CUDA : EXCL_OK;
        if (!launch_failed) {
            cudaError_t e;
            while ((e = cudaEventQuery(sl->done)) == cudaErrorNotReady) std::this_thread::yield();
            if (e != cudaSuccess) status = EXCL_E_CUDA;
        }
        const Clock::time_point t = Clock::now();
        if (!status) status = fail_status(*(volatile uint32_t *)sl->h_err);
        const uint32_t nq = (uint32_t)sl->batch.size();
        // results out of the mapped buffers before the slot is reused
        if (!status)
            for (uint32_t i = 0; i < nq; ++i) {
                Request &r = *sl->batch[i];
                const uint32_t o0 = sl->h_offsets[i], o1 = sl->h_offsets[i + 1];
                const uint32_t *d = sl->h_docids + o0;
                const uint32_t n = o1 - o0;
                if (r.replay) {
                    if (!n) r.replay->cs0.fetch_add(1);
                    else {
                        r.replay->cs1.fetch_add(n);
                        r.replay->cs2.fetch_xor((uint64_t)(d[0] ^ d[n - 1] ^ d[n / 2]));
                    }
                } else {
                    r.result.assign(d, d + n);
                }
            }
        {
            std::lock_guard<std::mutex> g(s->mu);
            for (auto &r : sl->batch) finish_locked(s, r, status, t);
            sl->batch.clear();
            s->pool.release(sl->pool_off, sl->pool_bytes);
            s->pool_in_use -= sl->pool_bytes;
            --s->inflight;
            if (status == EXCL_E_CUDA && !s->sticky) s->sticky = status;
            std::lock_guard<std::mutex> g2(sl->mu);
            sl->has_work = false;
            sl->busy = false;
        }
        s->cv_done.notify_all();
        s->cv_dispatch.notify_one();
    }
}

// Builds a request (no lock held): validates the terms and finds the
// shortest list, the first of equal lengths as the batch kernel's stable sort.
int make_request(excl_server *s, const uint32_t *terms, uint32_t nterms, ReqPtr *out) {
    if (nterms > kMaxTerms || (!terms && nterms)) return EXCL_E_INVALID;
    auto r = std::make_shared<Request>();
    r->terms.assign(terms, terms + nterms);
    uint32_t best = 0xffffffffu;
    for (uint32_t i = 0; i < nterms; ++i) {
        const uint32_t t = terms[i];
        if (t >= s->ix->nlists) return EXCL_E_INVALID;
        if (best == 0xffffffffu || s->ix->lists[t].n < s->ix->lists[best].n) best = t;
    }
    if (nterms) {
        r->keys = s->ix->lists[best].n;
        r->tiles = s->ix->lists[best].ntiles;
    }
    *out = std::move(r);
    return EXCL_OK;
}

// Queues requests in order under one lock; tickets only for the caller-waited ones.
int enqueue(excl_server *s, ReqPtr *reqs, size_t n, uint64_t *ticket) {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return EXCL_E_INVALID;
    if (s->sticky) return s->sticky;
    for (size_t i = 0; i < n; ++i) {
        ReqPtr &r = reqs[i];
        r->id = s->next_id++;
        if (!r->replay) s->tickets[r->id] = r;
        if (ticket) *ticket = r->id;
        s->queue.push_back(std::move(r));
    }
    s->submitted += n;
    return EXCL_OK;
}

void server_free(excl_server *s) {
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_dispatch.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    // in-flight batches finish; then the slot threads end
    {
        std::unique_lock<std::mutex> g(s->mu);
        s->cv_done.wait(g, [&] { return s->inflight == 0; });
        s->stop_slots = true;
    }
    for (auto &sl : s->slots) {
        {
            std::lock_guard<std::mutex> g(sl->mu);
        }
        sl->cv.notify_all();
        if (sl->worker.joinable()) sl->worker.join();
    }
    cudaSetDevice(s->device);
    for (auto &sl : s->slots) {
        if (sl->stream) cudaStreamSynchronize(sl->stream);
        cudaFree(sl->d_sync);
        cudaFree(sl->d_chunk);
        cudaFree(sl->d_misc);
        cudaFreeHost(sl->h_terms);
        cudaFreeHost(sl->h_toff);
        cudaFreeHost(sl->h_err);
        cudaFreeHost(sl->h_offsets);
        cudaFreeHost(sl->h_docids);
        if (sl->done) cudaEventDestroy(sl->done);
        if (sl->stream) cudaStreamDestroy(sl->stream);
    }
    cudaFree(s->d_pool);
    delete s;
}

}  // namespace

extern "C" int excl_server_create(int device, excl_index *ix, const excl_server_config *cfg, excl_server **out) {
    if (!ix || !out) return EXCL_E_INVALID;
    *out = nullptr;
    if (!ix->dev || ix->dev->device != device) return EXCL_E_INVALID;  // upload the index to this device first
    excl_server *s = new (std::nothrow) excl_server();
    if (!s) return EXCL_E_NOMEM;
    s->device = device;
    s->ix = ix;
    excl_server_config c{};
    if (cfg) c = *cfg;
    if (c.slots == 0) c.slots = 4;
    if (c.slots > 64) c.slots = 64;
    if (c.max_batch_queries == 0 || c.max_batch_queries > kPackMaxQueries) c.max_batch_queries = 4096;
    if (c.max_batch_keys == 0) c.max_batch_keys = 1ull << 22;
    if (c.max_batch_keys > 0xffffffffull / 2) c.max_batch_keys = 0xffffffffull / 2;
    if (c.algo > EXCL_ALGO_SEGREG) c.algo = EXCL_ALGO_AUTO;
    s->slot_max_tiles = (uint32_t)(c.max_batch_keys / kMinBlock + c.max_batch_queries + 1);
    const uint64_t per_batch =
        ws_layout(c.max_batch_queries, (uint64_t)c.max_batch_queries * 8, s->slot_max_tiles, c.max_batch_keys).total;
    if (c.hbm_budget_bytes == 0) c.hbm_budget_bytes = per_batch * c.slots;
    s->cfg = c;
    s->pool_size = up256(c.hbm_budget_bytes);
    s->pool.init(s->pool_size);
    int st = EXCL_OK;
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && !st) st = e == cudaErrorMemoryAllocation ? EXCL_E_NOMEM : EXCL_E_CUDA;
    };
    ck(cudaSetDevice(device));
    ck(cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, device));
    ck(cudaMalloc(&s->d_pool, s->pool_size));
    const size_t nchunk = s->slot_max_tiles / kSSChunk + 2;
    for (uint32_t i = 0; i < c.slots && !st; ++i) {
        auto sl = std::make_unique<Slot>();
        ck(cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking));
        ck(cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming));
        ck(cudaMalloc(&sl->d_sync, sizeof(PackSync)));
        ck(cudaMalloc(&sl->d_chunk, nchunk * 8));
        ck(cudaMalloc(&sl->d_misc, 256));
        ck(cudaHostAlloc(&sl->h_terms, (size_t)c.max_batch_queries * kMaxTerms * 4, cudaHostAllocMapped));
        ck(cudaHostAlloc(&sl->h_toff, ((size_t)c.max_batch_queries + 1) * 4, cudaHostAllocMapped));
        ck(cudaHostAlloc(&sl->h_err, 64, cudaHostAllocMapped));
        ck(cudaHostAlloc(&sl->h_offsets, ((size_t)c.max_batch_queries + 1) * 4, cudaHostAllocMapped));
        ck(cudaHostAlloc(&sl->h_docids, (size_t)c.max_batch_keys * 4, cudaHostAllocMapped));
        if (!st) {
            ck(cudaHostGetDevicePointer((void **)&sl->m_offsets, sl->h_offsets, 0));
            ck(cudaHostGetDevicePointer((void **)&sl->m_docids, sl->h_docids, 0));
            ck(cudaHostGetDevicePointer((void **)&sl->m_terms, sl->h_terms, 0));
            ck(cudaHostGetDevicePointer((void **)&sl->m_toff, sl->h_toff, 0));
            ck(cudaHostGetDevicePointer((void **)&sl->m_err, sl->h_err, 0));
            ck(cudaMemset(sl->d_sync, 0, sizeof(PackSync)));
            ck(cudaMemset(sl->d_chunk, 0, nchunk * 8));
            ck(cudaMemset(sl->d_misc, 0, 256));
        }
        s->slots.push_back(std::move(sl));
    }
    if (!st) ck(cudaDeviceSynchronize());
    if (st) {
        server_free(s);
        return st;
    }
    for (auto &sl : s->slots) sl->worker = std::thread(slot_loop, s, sl.get());
    s->dispatcher = std::thread(dispatch_loop, s);
    *out = s;
    return EXCL_OK;
}

extern "C" int excl_server_destroy(excl_server *s) {
    if (!s) return EXCL_E_INVALID;
    server_free(s);
    return EXCL_OK;
}

extern "C" int excl_server_submit(excl_server *s, const uint32_t *terms, uint32_t nterms, uint64_t *ticket) {
    if (!s || !ticket) return EXCL_E_INVALID;
    ReqPtr r;
    int st = make_request(s, terms, nterms, &r);
    if (st) return st;
    r->t_submit = Clock::now();
    st = enqueue(s, &r, 1, ticket);
    if (!st) s->cv_dispatch.notify_one();
    return st;
}

extern "C" int excl_server_wait(excl_server *s, uint64_t ticket, uint32_t *docids, size_t cap, uint32_t *n,
                                int timeout_ms) {
    if (!s) return EXCL_E_INVALID;
    std::unique_lock<std::mutex> g(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return EXCL_E_INVALID;
    ReqPtr r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) s->cv_done.wait(g, ready);
    else if (!s->cv_done.wait_for(g, std::chrono::milliseconds(timeout_ms), ready)) return EXCL_E_TIMEOUT;
    const size_t cnt = r->result.size();
    if (n) *n = (uint32_t)cnt;
    if (r->status) {
        s->tickets.erase(ticket);
        return r->status;
    }
    if (cnt > cap || (!docids && cnt)) return EXCL_E_CAPACITY;  // ticket kept: retry with a larger buffer
    if (cnt) std::memcpy(docids, r->result.data(), cnt * 4);
    s->tickets.erase(ticket);
    return EXCL_OK;
}

extern "C" int excl_server_stats_get(excl_server *s, excl_server_stats *out) {
    if (!s || !out) return EXCL_E_INVALID;
    std::vector<float> lat;
    {
        std::lock_guard<std::mutex> g(s->mu);
        std::memset(out, 0, sizeof *out);
        out->submitted = s->submitted;
        out->completed = s->completed;
        out->batches = s->batches;
        out->rejected = s->rejected;
        out->mean_batch = s->batches ? (double)(s->completed) / (double)s->batches : 0.0;
        out->pool_bytes = s->pool_size;
        out->pool_peak_bytes = s->pool_peak;
        out->max_inflight = s->max_inflight;
        lat = s->lat_us;
    }
    if (!lat.empty()) {
        auto pct = [&](double p) {
            const size_t k = std::min(lat.size() - 1, (size_t)(p * (double)(lat.size() - 1) + 0.5));
            std::nth_element(lat.begin(), lat.begin() + k, lat.end());
            return (double)lat[k];
        };
        out->p50_us = pct(0.50);
        out->p99_us = pct(0.99);
        out->max_us = *std::max_element(lat.begin(), lat.end());
    }
    return EXCL_OK;
}

extern "C" int excl_server_stats_reset(excl_server *s) {
    if (!s) return EXCL_E_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    s->lat_us.clear();
    s->submitted = s->completed = s->batches = s->rejected = 0;
    s->pool_peak = s->pool_in_use;
    s->max_inflight = s->inflight;
    return EXCL_OK;
}

extern "C" int excl_server_replay(excl_server *s, const uint32_t *terms, const uint32_t *term_offsets, uint32_t nq,
                                  const double *arrival_s, double *latency_s, uint64_t cs[3], double *wall_s) {
    if (!s || !term_offsets || !arrival_s || (!terms && term_offsets[nq] != term_offsets[0])) return EXCL_E_INVALID;
    for (uint32_t q = 0; q < nq; ++q) {
        if (term_offsets[q + 1] < term_offsets[q] || term_offsets[q + 1] - term_offsets[q] > kMaxTerms)
            return EXCL_E_INVALID;
        for (uint32_t i = term_offsets[q]; i < term_offsets[q + 1]; ++i)
            if (terms[i] >= s->ix->nlists) return EXCL_E_INVALID;
    }
    Replay rp;
    rp.latency_s = latency_s;
    rp.remaining.store(nq);
    const Clock::time_point t0 = Clock::now();
    auto due = [&](uint32_t q) {
        return t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[q]));
    };
    std::vector<ReqPtr> reqs;
    uint32_t q = 0;
    while (q < nq) {
        Clock::time_point now = Clock::now();
        if (now < due(q)) {
            const auto wait = due(q) - now;
            if (wait > std::chrono::microseconds(200)) std::this_thread::sleep_for(wait - std::chrono::microseconds(100));
            else std::this_thread::yield();
            continue;
        }
        // every query already due goes in under one lock; its latency counts
        // from its scheduled arrival, so a late submit is not hidden
        reqs.clear();
        uint32_t qe = q;
        while (qe < nq && due(qe) <= now) {
            ReqPtr r;
            const int st = make_request(s, terms + term_offsets[qe], term_offsets[qe + 1] - term_offsets[qe], &r);
            if (st) return st;  // validated above
            r->replay = &rp;
            r->replay_q = qe;
            r->t_submit = due(qe);
            reqs.push_back(std::move(r));
            ++qe;
        }
        const int st = enqueue(s, reqs.data(), reqs.size(), nullptr);
        if (st) {
            rp.status.store(st);
            rp.remaining.fetch_sub(nq - q);
            break;
        }
        s->cv_dispatch.notify_one();
        q = qe;
    }
    while (rp.remaining.load() != 0) std::this_thread::sleep_for(std::chrono::microseconds(50));
    if (wall_s) *wall_s = std::chrono::duration<double>(Clock::now() - t0).count();
    if (cs) {
        cs[0] = rp.cs0.load();
        cs[1] = rp.cs1.load();
        cs[2] = rp.cs2.load();
    }
    return rp.status.load();
}
