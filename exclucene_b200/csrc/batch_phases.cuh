// Pack and scatter phases of the one-launch batch kernel (k_batch in
// kernels.cu). A batch is one persistent grid that runs three phases:
//
//   pack     CTAs take chunks of 256 queries by ticket. Per query: sort the
//            terms by list length (stable insertion sort,
//            ParaPFD_Intersection.cu:155-173), count the shortest list's
//            tiles, docIDs and heavy tiles; a block scan plus a decoupled
//            look-back over the chunks give the batch's prefixes; each tile's
//            16-byte work record goes to its place in the probe order (heavy
//            tiles from the front, the others from the back). The chunk that
//            finishes last publishes the batch's "packed" tag.
//   probe    kernels.cu: warps take work records from a counter.
//   scatter  once every taken tile is probed (a count the probe warps add to
//            once each as they leave the probe loop), CTAs take chunks of 512
//            tiles: survivor totals, a decoupled look-back for their base,
//            each tile's output position (replaces cudppScan and ucntResult,
//            ParaPFD_Intersection.cu:262,301); then every warp copies
//            survivors to the result array (replaces saCompact, :279) and
//            every thread writes query offsets.
//
// Every wait is on work that a running CTA already holds (a ticket it took,
// tiles it took), so the grid needs no co-residency and batches on other
// streams may share the GPU. Cross-CTA state carries the batch's tag and is
// never cleared between batches; the counters are reset by the last CTA to
// leave. Every wait is bounded and raises kErrScanSpin when it gives up.
#pragma once
#include "kernels.h"

namespace excl {

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release64(uint64_t *p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_acquire64(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(uint32_t *p, uint32_t v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr uint32_t kPackRegTerms = 8;  // queries with up to this many terms are sorted in registers

// Batch tags cycle through 1 .. 2^30 - 1 (0 is the state of fresh memory).
__device__ __forceinline__ uint32_t next_tag(uint32_t e) { return e >= (1u << 30) - 1u ? 1u : e + 1u; }

// Chunk state of the scatter look-back: tag (30 bits) | status (2 bits) | value (32 bits).
constexpr uint32_t kAggregate = 1u, kPrefix = 2u;
__device__ __forceinline__ uint64_t chunk_word(uint32_t tag, uint32_t status, uint32_t v) {
    return ((uint64_t)tag << 34) | ((uint64_t)status << 32) | v;
}

// Bounded wait until *p == tag (acquire); false (and kErrScanSpin) if it gave up.
__device__ __forceinline__ bool wait_tag(const uint32_t *p, uint32_t tag, uint32_t *err, uint32_t spin) {
    uint32_t spins = 0;
    while (ld_acquire(p) != tag) {
        if (++spins > spin) {
            atomicOr(err, kErrScanSpin);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// Shared memory of the pack and scatter phases (a union with the probe's).
struct PackShared {
    uint32_t sc[3][33], pre[3], et[kPackThreads], eh[kPackThreads], h[kPackThreads], l0[kPackThreads];
};
struct ScatterShared {
    uint32_t sa[33], sb[33];
    uint32_t c, base;
};

// Block-wide exclusive scan of three values at once; returns the block totals.
__device__ __forceinline__ void block_scan3(const uint32_t (&v)[3], uint32_t (&e)[3], uint32_t (&t)[3],
                                            uint32_t (*sh)[33]) {
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t in[3] = {v[0], v[1], v[2]};
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, in[j], o);
            if (lane >= (uint32_t)o) in[j] += x;
        }
    if (lane == 31)
#pragma unroll
        for (int j = 0; j < 3; ++j) sh[j][w] = in[j];
    __syncthreads();
    if (w == 0) {
        uint32_t a[3], c[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) c[j] = a[j] = lane < nw ? sh[j][lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const uint32_t x = __shfl_up_sync(0xffffffffu, c[j], o);
                if (lane >= (uint32_t)o) c[j] += x;
            }
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (lane < nw) sh[j][lane] = c[j] - a[j];
            if (lane == 31) sh[j][32] = c[j];
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        e[j] = sh[j][w] + in[j] - v[j];
        t[j] = sh[j][32];
    }
}

// Block-wide exclusive scan of one value; returns the block total.
__device__ __forceinline__ uint32_t block_scan1(uint32_t a, uint32_t &total, uint32_t *sa) {
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t ia = a;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t xa = __shfl_up_sync(0xffffffffu, ia, o);
        if (lane >= (uint32_t)o) ia += xa;
    }
    if (lane == 31) sa[w] = ia;
    __syncthreads();
    if (w == 0) {
        const uint32_t va = lane < nw ? sa[lane] : 0u;
        uint32_t ja = va;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t xa = __shfl_up_sync(0xffffffffu, ja, o);
            if (lane >= (uint32_t)o) ja += xa;
        }
        if (lane < nw) sa[lane] = ja - va;
        if (lane == 31) sa[32] = ja;
    }
    __syncthreads();
    const uint32_t ex = sa[w] + ia - a;
    total = sa[32];
    __syncthreads();  // sa is reused by the caller's next scan
    return ex;
}

// Tiles of a query's shortest list that hold at least half a tile of keys:
// the first `heavy` tiles (all full tiles, and the last one when it is at
// least half full). A tile's probe time grows with its keys, so these go to
// the front of the probe order and the small tiles fill the end (longest
// first keeps the busiest SM near the average). Variable (HS) tiles all count
// as heavy.
__device__ __forceinline__ uint32_t heavy_tiles(uint32_t n, uint32_t nt, uint32_t log2_block, uint32_t split) {
    if (!log2_block || nt == 0) return nt;
    const uint32_t S = (1u << log2_block) >> tile_split_of(log2_block, split);
    return min(nt, n / S + (2u * (n % S) >= S ? 1u : 0u));
}

// Pack chunk `bid` of `npack` (queries bid*256 .. +255) with the CTA's 256
// threads. The chunk that completes last finishes the phase: batch totals are
// out (the last chunk wrote them), the probe counter and statistics are
// cleared, and sync->packed = tag releases the probe phase.
__device__ __noinline__ void pack_chunk(uint32_t bid, uint32_t npack, uint32_t tag, const ListDesc *__restrict__ lists,
                                           uint32_t nlists, const uint32_t *terms, const uint32_t *toff, uint32_t nq,
                                           const BatchView &b, PackSync *__restrict__ sync, PackShared &sm,
                                           uint32_t spin) {
    const uint32_t q = bid * kPackThreads + threadIdx.x;
    uint32_t nt = 0, nk = 0, lb0 = 0, l0 = 0;
    if (q < nq) {
        const uint32_t t0 = toff[q], t1 = toff[q + 1];
        uint32_t k = t1 >= t0 ? t1 - t0 : 0u;
        if (k > kMaxTerms) {
            atomicOr(b.err, kErrTerms);
            k = 0;
        }
        uint32_t *dst = const_cast<uint32_t *>(b.qterms) + (size_t)q * kMaxTerms;
        if (k <= kPackRegTerms) {
            // common case: all in registers, every load of the query issued at once
            uint32_t id[kPackRegTerms], len[kPackRegTerms], ntl[kPackRegTerms], lbl[kPackRegTerms];
            bool bad = false;
#pragma unroll
            for (uint32_t j = 0; j < kPackRegTerms; ++j) id[j] = j < k ? terms[t0 + j] : 0u;
#pragma unroll
            for (uint32_t j = 0; j < kPackRegTerms; ++j) {
                const bool v = j < k && id[j] < nlists;
                bad |= j < k && id[j] >= nlists;
                len[j] = v ? __ldg(&lists[id[j]].n) : 0xffffffffu;  // absent terms sort last
                lbl[j] = v ? __ldg(&lists[id[j]].log2_block) : 0u;
                ntl[j] = v ? split_tiles(len[j], __ldg(&lists[id[j]].ntiles), lbl[j], b.tile_split) : 0u;
            }
            if (bad) {
                atomicOr(b.err, kErrTermId);
                k = 0;
            }
            // stable insertion sort by length with fixed indices (strict compare keeps input order on ties)
#pragma unroll
            for (uint32_t i = 1; i < kPackRegTerms; ++i)
#pragma unroll
                for (uint32_t j = i; j > 0; --j)
                    if (len[j] < len[j - 1]) {
                        uint32_t x = id[j]; id[j] = id[j - 1]; id[j - 1] = x;
                        x = len[j]; len[j] = len[j - 1]; len[j - 1] = x;
                        x = ntl[j]; ntl[j] = ntl[j - 1]; ntl[j - 1] = x;
                        x = lbl[j]; lbl[j] = lbl[j - 1]; lbl[j - 1] = x;
                    }
#pragma unroll
            for (uint32_t j = 0; j < kPackRegTerms; ++j)
                if (j < k) dst[j] = id[j];
            nt = k ? ntl[0] : 0u;
            nk = k ? len[0] : 0u;
            lb0 = k ? lbl[0] : 0u;
            l0 = k ? id[0] : 0u;
        } else {
            uint32_t id[kMaxTerms], len[kMaxTerms];
            bool bad = false;
            // loads in groups of four so their latencies overlap
            for (uint32_t i0 = 0; i0 < k; i0 += 4) {
#pragma unroll
                for (uint32_t j = 0; j < 4; ++j)
                    if (i0 + j < k) id[i0 + j] = terms[t0 + i0 + j];
            }
            for (uint32_t i0 = 0; i0 < k; i0 += 4) {
#pragma unroll
                for (uint32_t j = 0; j < 4; ++j)
                    if (i0 + j < k) {
                        const uint32_t tid = id[i0 + j];
                        bad |= tid >= nlists;
                        len[i0 + j] = tid < nlists ? __ldg(&lists[tid].n) : 0u;
                    }
            }
            if (bad) {
                atomicOr(b.err, kErrTermId);
                k = 0;
            }
            for (uint32_t i = 1; i < k; ++i) {
                const uint32_t ci = id[i], cl = len[i];
                uint32_t j = i;
                while (j && cl < len[j - 1]) {
                    id[j] = id[j - 1];
                    len[j] = len[j - 1];
                    --j;
                }
                id[j] = ci;
                len[j] = cl;
            }
            for (uint32_t i = 0; i < k; ++i) dst[i] = id[i];
            lb0 = k ? __ldg(&lists[id[0]].log2_block) : 0u;
            nt = k ? split_tiles(len[0], __ldg(&lists[id[0]].ntiles), lb0, b.tile_split) : 0u;
            nk = k ? len[0] : 0u;
            l0 = k ? id[0] : 0u;
        }
        const_cast<uint32_t *>(b.qnterms)[q] = k;
    }
    const uint32_t nh = heavy_tiles(nk, nt, lb0, b.tile_split);
    uint32_t ex[3], tot[3];
    block_scan3({nt, nk, nh}, ex, tot, sm.sc);
    const uint32_t et = ex[0], ek = ex[1], bt = tot[0], bk = tot[1];
    if (threadIdx.x == 0) {
        sync->agg_t[bid] = bt;
        sync->agg_k[bid] = bk;
        sync->agg_h[bid] = tot[2];
        st_release(&sync->flag[bid], tag);
    }
    if (threadIdx.x < 32) {
        // warp 0: the predecessors' totals. Every predecessor took its ticket
        // earlier, so it is running or done. Each lane has the flags of four
        // predecessors in flight at once; one fence then orders the totals'
        // loads after the flags that published them.
        const uint32_t lane = threadIdx.x;
        uint32_t pt = 0, pk = 0, ph = 0;
        for (uint32_t p0 = 0; p0 < bid; p0 += 128) {
            uint32_t f[4];
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j) {
                const uint32_t p = p0 + lane + 32u * j;
                f[j] = p < bid ? ld_relaxed(&sync->flag[p]) : tag;
            }
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j) {
                const uint32_t p = p0 + lane + 32u * j;
                uint32_t spins = 0;
                while (f[j] != tag) {
                    if (++spins > spin) {
                        atomicOr(b.err, kErrScanSpin);
                        break;
                    }
                    __nanosleep(32);
                    f[j] = ld_relaxed(&sync->flag[p]);
                }
            }
            __threadfence();
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j) {
                const uint32_t p = p0 + lane + 32u * j;
                if (p < bid) {
                    pt += ld_relaxed(&sync->agg_t[p]);
                    pk += ld_relaxed(&sync->agg_k[p]);
                    ph += ld_relaxed(&sync->agg_h[p]);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            pt += __shfl_xor_sync(0xffffffffu, pt, o);
            pk += __shfl_xor_sync(0xffffffffu, pk, o);
            ph += __shfl_xor_sync(0xffffffffu, ph, o);
        }
        if (lane == 0) {
            sm.pre[0] = pt;
            sm.pre[1] = pk;
            sm.pre[2] = ph;
        }
    }
    sm.et[threadIdx.x] = et;
    sm.eh[threadIdx.x] = ex[2];
    sm.h[threadIdx.x] = nh;
    sm.l0[threadIdx.x] = l0;
    __syncthreads();
    const uint32_t pt = sm.pre[0];
    if (threadIdx.x == 0 && bid == npack - 1) {
        const uint32_t pk = sm.pre[1];
        const_cast<uint32_t *>(b.tile_prefix)[nq] = pt + bt;
        const_cast<uint32_t *>(b.tile_prefix)[nq + 1] = sm.pre[2] + tot[2];  // heavy tiles in the batch
        const_cast<uint32_t *>(b.key_base)[nq] = pk + bk;
        if ((uint64_t)pt + bt > b.max_tiles || (uint64_t)pk + bk > b.max_keys) atomicOr(b.err, kErrCapacity);
    }
    if (q < nq) {
        const_cast<uint32_t *>(b.tile_prefix)[q] = pt + et;
        const_cast<uint32_t *>(b.key_base)[q] = sm.pre[1] + ek;
    }
    // owner of each of this CTA's tiles: the last query whose first tile is
    // at or before it (queries with no tiles share their successor's start);
    // its work record goes to its place in the probe order: heavy tiles from
    // the front in query order, the others from the back of tile_order
    // (a thread's tiles ascend, so its owners do too: the search resumes from
    // the last owner, and a run of one query's tiles costs one check each)
    const uint32_t ph = sm.pre[2];
    uint32_t lo = 0;
    for (uint32_t tl = threadIdx.x; tl < bt && pt + tl < b.max_tiles; tl += blockDim.x) {
        if (lo + 1 < blockDim.x && sm.et[lo + 1] <= tl) {
            uint32_t hi = blockDim.x - 1;
            ++lo;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (sm.et[mid] <= tl) lo = mid;
                else hi = mid - 1;
            }
        }
        const uint32_t t = pt + tl, i = tl - sm.et[lo], hb = ph + sm.eh[lo];
        const uint4 wr = make_uint4(t, bid * blockDim.x + lo, i, sm.l0[lo]);
        if (i < sm.h[lo]) b.tile_order[hb + i] = wr;
        else b.tile_order[b.max_tiles - 1u - (t - hb - sm.h[lo])] = wr;
    }
    // this chunk is done once every thread's writes are visible; the chunk
    // that completes last releases the probe phase
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0 && atomicAdd(&sync->done, 1u) == npack - 1) {
        __threadfence();  // the other chunks' writes (ordered by their fence before counting) and the totals
        *b.tile_counter = 0u;
        *b.probe_done = 0u;
        if (b.stats) {
            b.stats[0] = b.stats[1] = b.stats[2] = b.stats[3] = b.stats[6] = 0ull;
            b.stats[5] = global_ns();
        }
        st_release(&sync->packed, tag);
    }
    __syncthreads();  // sm is reused by the next chunk
}

// The batch's error bits to the host word the batch names (the device word is
// cleared for the next batch); nothing when it names none.
__device__ __forceinline__ void hand_over_flags(const BatchView &b) {
    if (!b.err_out) return;
    *(volatile uint32_t *)b.err_out = atomicExch(b.err, 0u);
    __threadfence_system();
}

// Scatter phase, run by every CTA once its warps have left the probe loop.
// Phase A (CTAs holding a chunk ticket): survivor total of the chunk,
// decoupled look-back for its base, the absolute output position of each of
// its tiles (into tile_q), then the chunk's inclusive prefix. Phase B (every
// warp, once all chunk tickets are taken, so every chunk is owned by a running
// CTA): query offsets, and survivors copied tile by tile, each tile after its
// chunk's prefix is out.
__device__ __noinline__ void scatter_phase(const BatchView &b, PackSync *__restrict__ sync,
                                              uint64_t *__restrict__ chunk_state, uint32_t *__restrict__ offsets,
                                              uint32_t *__restrict__ docids, uint64_t cap, uint32_t tag,
                                              ScatterShared &sm, uint32_t spin) {
    constexpr uint32_t kPer = kSSChunk / kSSThreads;
    static_assert(kPer == 2, "two tiles per thread");
    const uint32_t nq = b.nq;
    const uint32_t T = min(b.tile_prefix[nq], b.max_tiles);
    const uint32_t nch = (T + kSSChunk - 1) / kSSChunk;
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t *tile_out = b.tile_q;
    if (nch == 0) {  // no tiles in the batch: every offset is 0
        for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q <= nq; q += gridDim.x * blockDim.x) offsets[q] = 0u;
        return;
    }
    for (;;) {
        if (threadIdx.x == 0) {
            sm.c = atomicAdd(&sync->sticket, 1u);
            // the chunk owners start once every tile of the batch is probed
            if (sm.c < nch) {
                uint32_t spins = 0;
                while (ld_acquire(b.probe_done) != T) {
                    if (++spins > spin) {
                        atomicOr(b.err, kErrScanSpin);
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __syncthreads();
        const uint32_t c = sm.c;
        if (c >= nch) break;
        const uint32_t t0 = c * kSSChunk;
        const uint32_t ta = t0 + threadIdx.x * kPer;
        const uint32_t c0 = ta < T ? b.tile_count[ta] : 0u;
        const uint32_t c1 = ta + 1 < T ? b.tile_count[ta + 1] : 0u;
        uint32_t tot;
        const uint32_t ex = block_scan1(c0 + c1, tot, sm.sa);
        if (threadIdx.x == 0) st_release64(&chunk_state[c], chunk_word(tag, kAggregate, tot));
        if (w == 0) {
            // look-back: sum the aggregates of the preceding chunks up to the
            // nearest one that has published its inclusive prefix
            uint32_t excl = 0;
            int64_t p = (int64_t)c - 1;
            for (;;) {
                const int64_t idx = p - (int64_t)lane;
                uint32_t st = kPrefix, v = 0;
                if (idx >= 0) {
                    uint64_t s = ld_acquire64(&chunk_state[idx]);
                    uint32_t spins = 0;
                    while ((uint32_t)(s >> 34) != tag) {
                        if (++spins > spin) {
                            atomicOr(b.err, kErrScanSpin);
                            s = chunk_word(tag, kPrefix, 0u);
                            break;
                        }
                        __nanosleep(32);
                        s = ld_acquire64(&chunk_state[idx]);
                    }
                    st = (uint32_t)(s >> 32) & 3u;
                    v = (uint32_t)s;
                }
                const uint32_t m = __ballot_sync(0xffffffffu, st == kPrefix);
                const uint32_t stop = m ? (uint32_t)(__ffs(m) - 1) : 31u;
                uint32_t contrib = lane <= stop ? v : 0u;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
                excl += contrib;
                if (m) break;
                p -= 32;
            }
            if (lane == 0) sm.base = excl;
        }
        __syncthreads();
        const uint32_t base = sm.base;
        if (ta < T) tile_out[ta] = base + ex;
        if (ta + 1 < T) tile_out[ta + 1] = base + ex + c0;
        if (c == nch - 1 && threadIdx.x == 0 && (uint64_t)base + tot > cap) atomicOr(b.err, kErrCapacity);
        __syncthreads();  // tile positions written before the prefix goes out
        if (threadIdx.x == 0) {
            __threadfence();
            st_release64(&chunk_state[c], chunk_word(tag, kPrefix, base + tot));
        }
    }
    // the query offsets: the output position of each query's first tile, or
    // for a query with no tile after it, the batch's total (the last chunk's
    // inclusive prefix); each once its chunk's prefix is out
    for (uint32_t qq = blockIdx.x * blockDim.x + threadIdx.x; qq <= nq; qq += gridDim.x * blockDim.x) {
        const uint32_t tp = min(b.tile_prefix[qq], T);
        const uint32_t c = tp < T ? tp / kSSChunk : nch - 1u;
        uint64_t s = ld_acquire64(&chunk_state[c]);
        uint32_t spins = 0;
        while ((uint32_t)(s >> 34) != tag || ((uint32_t)(s >> 32) & 3u) != kPrefix) {
            if (++spins > spin) {
                atomicOr(b.err, kErrScanSpin);
                break;
            }
            __nanosleep(64);
            s = ld_acquire64(&chunk_state[c]);
        }
        offsets[qq] = tp < T ? ld_acquire(&tile_out[tp]) : (uint32_t)s;
    }
    // survivors: warp w takes tiles w, w + nw, w + 2nw, ... (neighbouring
    // tiles go to different warps, so a query with many survivors spreads over
    // the grid). Lane j handles the warp's j-th tile of a round of 32: its
    // survivor count, its chunk's prefix (bounded wait), its output position
    // and slot, all lanes at once; then the warp copies the non-empty tiles
    // one after another, eight independent loads per lane.
    const uint32_t gw = blockIdx.x * (blockDim.x / 32) + w, nw = gridDim.x * (blockDim.x / 32);
    const uint32_t *__restrict__ scr = b.scratch;
    for (uint64_t j0 = 0; gw + j0 * nw < T; j0 += 32) {
        const uint64_t tt = gw + (j0 + lane) * nw;
        const uint32_t t = tt < T ? (uint32_t)tt : T;
        const uint32_t n = t < T ? b.tile_count[t] : 0u;
        uint32_t o = 0, slot = 0;
        if (n) {
            const uint32_t c = t / kSSChunk;
            uint64_t s = ld_acquire64(&chunk_state[c]);
            uint32_t spins = 0;
            while ((uint32_t)(s >> 34) != tag || ((uint32_t)(s >> 32) & 3u) != kPrefix) {
                if (++spins > spin) {
                    atomicOr(b.err, kErrScanSpin);
                    break;
                }
                __nanosleep(64);
                s = ld_acquire64(&chunk_state[c]);
            }
            o = ld_acquire(&tile_out[t]);
            slot = b.tile_slot[t];
        }
        uint32_t m = __ballot_sync(0xffffffffu, n != 0u);
        while (m) {
            const uint32_t l = (uint32_t)(__ffs(m) - 1);
            m &= m - 1u;
            const uint32_t nl = __shfl_sync(0xffffffffu, n, l), ol = __shfl_sync(0xffffffffu, o, l),
                           sl = __shfl_sync(0xffffffffu, slot, l);
            const uint32_t *src = scr + sl;
            uint32_t v[kTileKeys / 32];
#pragma unroll
            for (uint32_t i = 0; i < kTileKeys / 32; ++i) {
                const uint32_t k = lane + 32u * i;
                if (k < nl) v[i] = src[k];
            }
#pragma unroll
            for (uint32_t i = 0; i < kTileKeys / 32; ++i) {
                const uint32_t k = lane + 32u * i;
                if (k < nl && (uint64_t)ol + k < cap) docids[(uint64_t)ol + k] = v[i];
            }
        }
    }
}

}  // namespace excl
