// Allocation-free variant of excl_intersect_device.
//
// Who needs it: callers that must not allocate device memory when they issue
// queries — a host that hands the library a fixed memory budget and forbids
// cudaMalloc/cudaFree after start-up (so the device allocator never
// synchronises or fragments under load), code that runs where the caller owns
// every allocation, or an embedding that cannot create a context (an
// excl_ctx reserves its batch buffers with cudaMalloc). This entry point runs
// the same kernels as excl_intersect_device, but all of its per-batch scratch
// (sorted query terms, tile and key prefixes, tile owners and work order, per-tile counts,
// survivor slots, scan state, error flag) lives in one file-scope device array of fixed size.
//
// Limits: at most EXCL_NOALLOC_MAX_QUERIES queries per call and at most
// EXCL_NOALLOC_MAX_KEYS docIDs summed over the queries' shortest lists. The
// array takes 5,835,264 bytes (5.6 MiB) on every GPU that loads the library,
// until the process exits.
//
// Sharing: every call uses the same array and it keeps the last call's
// contents; each call clears what must start at zero (error flag, counters,
// scan state) on its stream. Calls whose work overlaps on the GPU (two
// streams, or two host threads) race on the array and must be serialised by
// the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "kernels.h"
#include "runtime.h"

namespace excl {
namespace {

constexpr uint32_t kNAQueries = EXCL_NOALLOC_MAX_QUERIES;
constexpr uint32_t kNAKeys = EXCL_NOALLOC_MAX_KEYS;
constexpr uint32_t kNATiles = kNAKeys / kMinBlock + kNAQueries + 1;  // bound as in ctx_alloc_batch

constexpr uint64_t up64(uint64_t w) { return (w + 63) & ~63ull; }  // regions start on 256-byte boundaries

// word offsets of the regions inside the array
constexpr uint64_t kOffQterms = 0;
constexpr uint64_t kOffQnterms = kOffQterms + up64((uint64_t)kNAQueries * kMaxTerms);
constexpr uint64_t kOffSync = kOffQnterms + up64(kNAQueries);        // PackSync
constexpr uint64_t kOffChunkState = kOffSync + up64(kNAQueries + 1);  // u64 look-back state per chunk
constexpr uint64_t kOffTilePrefix = kOffChunkState + up64(kNAQueries + 1);
constexpr uint64_t kOffKeyBase = kOffTilePrefix + up64(kNAQueries + 2);
constexpr uint64_t kOffTileQ = kOffKeyBase + up64(kNAQueries + 2);
constexpr uint64_t kOffTileCount = kOffTileQ + up64(kNATiles + 1);
constexpr uint64_t kOffTileSlot = kOffTileCount + up64(kNATiles + 1);
constexpr uint64_t kOffTileOrder = kOffTileSlot + up64(kNATiles + 1);
constexpr uint64_t kOffSurvivors = kOffTileOrder + up64(4 * ((uint64_t)kNATiles + 1));  // 16-byte work records
constexpr uint64_t kOffMisc = kOffSurvivors + up64(kNAKeys);
constexpr uint64_t kOffStats = kOffMisc + 64;           // 8 x u64: probes, fallbacks, keys, merges, phase times
constexpr uint64_t kWords = kOffStats + 64;
static_assert(sizeof(PackSync) <= 4 * (kOffChunkState - kOffSync), "pack state region");
static_assert(2 * (kNATiles / kSSChunk + 2) <= kOffTilePrefix - kOffChunkState, "chunk state region");
static_assert(kWords * 4 == 5835264, "scratch size stated in the comments and excl_gpu.h");

static __device__ __align__(256) uint32_t g_noalloc_scratch[kWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t *g_base[kMaxDevices];  // device address of g_noalloc_scratch, per device
int g_nsm[kMaxDevices];

// First call on a device (with that device current): look up the device
// address of the array. The host-side name g_noalloc_scratch is only a
// stand-in, never a device address, so kernels get this pointer instead.
// The batch pipeline's cross-CTA state must start zeroed (its tags start at
// 1). A file-scope device array is zero when the module loads; the state is
// cleared once more here, on the caller's stream so the clear is ordered
// before this first batch, in case the array was used before the lookup.
int setup_device(int dev, cudaStream_t st, uint32_t **base, int *nsm) {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_base[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return EXCL_E_CUDA;
        e = cudaMemsetAsync(static_cast<uint32_t *>(p) + kOffSync, 0, 4 * (kOffTilePrefix - kOffSync), st);
        if (e != cudaSuccess) return EXCL_E_CUDA;
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return EXCL_E_CUDA;
        g_nsm[dev] = n;
        g_base[dev] = static_cast<uint32_t *>(p);
    }
    *base = g_base[dev];
    *nsm = g_nsm[dev];
    return EXCL_OK;
}

}  // namespace
}  // namespace excl

using namespace excl;

extern "C" int excl_intersect_device_noalloc(excl_index *ix, const uint32_t *d_terms, const uint32_t *d_term_offsets,
                                             uint32_t nq, uint32_t algo, uint32_t *d_offsets, uint32_t *d_docids,
                                             uint64_t cap, void *stream) {
    if (!ix || !ix->dev || !d_term_offsets || !d_offsets || (!d_docids && cap) || algo > EXCL_ALGO_SEGREG)
        return EXCL_E_INVALID;
    if (nq > kNAQueries) return EXCL_E_CAPACITY;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return EXCL_E_CUDA;
    if (dev != ix->dev->device) return EXCL_E_INVALID;  // the index lives on another device
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t *base = nullptr;
    int nsm = 0;
    int s = setup_device(dev, st, &base, &nsm);
    if (s) return s;

    BatchView b{};
    b.nq = nq;
    b.qterms = base + kOffQterms;
    b.qnterms = base + kOffQnterms;
    b.tile_prefix = base + kOffTilePrefix;
    b.tile_q = base + kOffTileQ;
    b.tile_counter = base + kOffMisc + 1;
    b.key_base = base + kOffKeyBase;
    b.tile_count = base + kOffTileCount;
    b.tile_slot = base + kOffTileSlot;
    b.tile_order = reinterpret_cast<uint4 *>(base + kOffTileOrder);
    b.scratch = base + kOffSurvivors;
    b.max_tiles = kNATiles;
    b.merge_segs = 2;
    b.max_keys = kNAKeys;
    b.err = base + kOffMisc;
    b.probe_done = base + kOffMisc + 32;  // its own 128-byte line, apart from the queue head
    b.scatter_ready = base + kOffMisc + 48;
    b.stats = reinterpret_cast<uint64_t *>(base + kOffStats);
    BatchLaunch L{};
    L.ixv = ix->dev->view(ix->models ? model_view(ix->models) : ModelView{});
    L.lists = ix->dev->lists;
    L.nlists = ix->nlists;
    L.terms = d_terms;
    L.toff = d_term_offsets;
    L.b = b;
    L.sync = reinterpret_cast<PackSync *>(base + kOffSync);
    L.chunk_state = reinterpret_cast<uint64_t *>(base + kOffChunkState);
    L.offsets = d_offsets;
    L.docids = d_docids;
    L.cap = cap;
    L.algo = (int)algo;
    L.warps = 8;
    L.ctas_per_sm = 5;
    L.nsm = nsm;
    L.ev = nullptr;

    int e = (int)cudaMemsetAsync(base + kOffMisc, 0, 64 * 4, st);  // error flag
    e |= launch_batch(L, st);
    if (e) return EXCL_E_CUDA;
    // the device-side limits (keys, tiles, result capacity) surface here
    uint32_t flags = 0;
    if (cudaMemcpyAsync(&flags, base + kOffMisc, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return EXCL_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return EXCL_E_CUDA;
    if (flags & kErrCapacity) return EXCL_E_CAPACITY;
    if (flags & (kErrTermId | kErrTerms)) return EXCL_E_INVALID;
    if (flags) return EXCL_E_DEVICE_FLAG;
    return EXCL_OK;
}
