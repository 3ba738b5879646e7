// Pack and scatter phases of the one-launch batch kernel (k_batch in
// kernels.cu). A batch is one persistent grid that runs three phases:
//
//   pack     CTAs take chunks of 256 queries by ticket. Per query: sort the
//            terms by list length (stable insertion sort,
//            ParaPFD_Intersection.cu:155-173), count the shortest list's
//            tiles, docIDs and heavy tiles; a block scan plus a decoupled
//            look-back over the chunks give the batch's prefixes; each tile's
//            16-byte work record goes to its place in the probe order (heavy
//            tiles from the front, the others from the back). Each chunk
//            publishes a done flag; the probe phase waits for all of them.
//   probe    kernels.cu: warps take work records from a counter.
//   scatter  CTAs take chunks of 512 tiles; a chunk owner waits until every
//            tile is probed (a count the probe warps add to once each as they
//            leave the probe loop), then scans its survivor counts, finds its base
//            by a decoupled look-back (replaces cudppScan,
//            ParaPFD_Intersection.cu:262), writes the offsets of the queries
//            that start in the chunk (ucntResult, :301) and its tiles' output
//            positions, and counts itself ready; once every chunk is ready,
//            every warp of the grid copies survivors (saCompact, :279).
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

// Polls of a cross-CTA word sleep between reads, doubling from 32 ns up to a
// cap, so a poller that waits long (a CTA done with its work, waiting for the
// slowest) puts little load on the word's L2 slice, which the working CTAs
// also use.

// Batch tags cycle through 1 .. 2^30 - 1 (0 is the state of fresh memory).
__device__ __forceinline__ uint32_t next_tag(uint32_t e) { return e >= (1u << 30) - 1u ? 1u : e + 1u; }

// Chunk state of the scatter look-back: tag (30 bits) | status (2 bits) | value (32 bits).
constexpr uint32_t kAggregate = 1u, kPrefix = 2u;
__device__ __forceinline__ uint64_t chunk_word(uint32_t tag, uint32_t status, uint32_t v) {
    return ((uint64_t)tag << 34) | ((uint64_t)status << 32) | v;
}

// Bounded wait until *p == want, polled with relaxed loads (a poll touches
// only the word's L2 line; an acquire load per poll would also order, and so
// hold up, the poller's later loads each time); once the value is seen, one
// acquire load makes the writes published before it visible. false (and
// kErrScanSpin in *err) if it gave up.
// `cap_ns` bounds the sleep between polls: short where few CTAs poll, longer
// where the whole grid polls one word.
__device__ __forceinline__ bool wait_eq(const uint32_t *p, uint32_t want, uint32_t *err, uint32_t spin,
                                        uint32_t cap_ns = 1024u) {
    uint32_t spins = 0, ns = 32;
    for (;;) {
        while (ld_relaxed(p) != want) {
            if (++spins > spin) {
                atomicOr(err, kErrScanSpin);
                return false;
            }
            __nanosleep(ns);
            ns = ns < cap_ns ? ns * 2u : cap_ns;
        }
        if (ld_acquire(p) == want) return true;
    }
}

// Bounded wait until *p == tag (the failure-path self-test's flag).
__device__ __forceinline__ bool wait_tag(const uint32_t *p, uint32_t tag, uint32_t *err, uint32_t spin) {
    return wait_eq(p, tag, err, spin);
}

// Shared memory of the pack and scatter phases (a union with the probe's).
struct PackShared {
    uint32_t sc[3][33], pre[3], et[kPackThreads], eh[kPackThreads], h[kPackThreads], l0[kPackThreads];
};
struct ScatterShared {
    uint32_t sa[33];
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

// Pack chunk `bid` of `npack` (queries bid*qpc .. +qpc-1, one per thread of
// the first qpc threads; the CTA's other threads take part in its scans and
// record writes). Its flag goes to tag << 1 once its aggregates are out (for
// the look-back of later chunks), and it counts itself in sync->packed once
// all its writes are visible; the last chunk also writes the batch totals,
// chunk 0 clears the probe phase's counters and the statistics.
__device__ __noinline__ void pack_chunk(uint32_t bid, uint32_t npack, uint32_t qpc, uint32_t tag,
                                           const ListDesc *__restrict__ lists, uint32_t nlists, const uint32_t *terms,
                                           const uint32_t *toff, uint32_t nq, const BatchView &b,
                                           PackSync *__restrict__ sync, PackShared &sm, uint32_t spin) {
    const uint32_t q = threadIdx.x < qpc ? bid * qpc + threadIdx.x : nq;
    uint32_t nt = 0, nk = 0, lb0 = 0, l0 = 0;
    // sorted terms of a query of <= kPackRegTerms terms, written only after
    // this chunk's aggregates are published (a release waits for its warp's
    // earlier writes)
    uint32_t idr[kPackRegTerms];
    uint32_t kreg = 0;
    bool regq = false;
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
                // n, ntiles and log2_block: the descriptor's first 16 bytes
                const uint4 m = v ? __ldg(reinterpret_cast<const uint4 *>(lists + id[j])) : make_uint4(0, 0, 0, 0);
                len[j] = v ? m.x : 0xffffffffu;  // absent terms sort last
                lbl[j] = m.z;
                ntl[j] = v ? split_tiles(m.x, m.y, m.z, b.tile_split) : 0u;
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
            for (uint32_t j = 0; j < kPackRegTerms; ++j) idr[j] = id[j];
            kreg = k;
            regq = true;
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
            const_cast<uint32_t *>(b.qnterms)[q] = k;
            lb0 = k ? __ldg(&lists[id[0]].log2_block) : 0u;
            nt = k ? split_tiles(len[0], __ldg(&lists[id[0]].ntiles), lb0, b.tile_split) : 0u;
            nk = k ? len[0] : 0u;
            l0 = k ? id[0] : 0u;
        }
    }
    const uint32_t nh = heavy_tiles(nk, nt, lb0, b.tile_split);
    uint32_t ex[3], tot[3];
    block_scan3({nt, nk, nh}, ex, tot, sm.sc);
    const uint32_t et = ex[0], ek = ex[1], bt = tot[0], bk = tot[1];
    if (threadIdx.x == 0) {
        sync->agg_t[bid] = bt;
        sync->agg_k[bid] = bk;
        sync->agg_h[bid] = tot[2];
        st_release(&sync->flag[bid], tag << 1);  // aggregates out
    }
    if (regq) {
        uint32_t *dst = const_cast<uint32_t *>(b.qterms) + (size_t)q * kMaxTerms;
#pragma unroll
        for (uint32_t j = 0; j < kPackRegTerms; ++j)
            if (j < kreg) dst[j] = idr[j];
        const_cast<uint32_t *>(b.qnterms)[q] = kreg;
    }
    {
        // the predecessors' totals, one predecessor per thread (all acquire
        // loads in flight at once), then a block reduction. Every predecessor
        // took its ticket earlier, so it is running or done.
        uint32_t pt = 0, pk = 0, ph = 0;
        for (uint32_t p = threadIdx.x; p < bid; p += blockDim.x) {
            uint32_t f = ld_acquire(&sync->flag[p]), spins = 0;
            while ((f >> 1) != tag) {  // aggregates not out yet
                if (++spins > spin) {
                    atomicOr(b.err, kErrScanSpin);
                    break;
                }
                __nanosleep(32);
                f = ld_acquire(&sync->flag[p]);
            }
            pt += ld_relaxed(&sync->agg_t[p]);
            pk += ld_relaxed(&sync->agg_k[p]);
            ph += ld_relaxed(&sync->agg_h[p]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            pt += __shfl_xor_sync(0xffffffffu, pt, o);
            pk += __shfl_xor_sync(0xffffffffu, pk, o);
            ph += __shfl_xor_sync(0xffffffffu, ph, o);
        }
        const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
        if (lane == 0) {
            sm.sc[0][w] = pt;
            sm.sc[1][w] = pk;
            sm.sc[2][w] = ph;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            uint32_t v = 0;
            for (uint32_t i = 0; i < (blockDim.x >> 5); ++i) v += sm.sc[threadIdx.x][i];
            sm.pre[threadIdx.x] = v;
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
        const uint4 wr = make_uint4(t, bid * qpc + lo, i, sm.l0[lo]);
        if (i < sm.h[lo]) b.tile_order[hb + i] = wr;
        else b.tile_order[b.max_tiles - 1u - (t - hb - sm.h[lo])] = wr;
    }
    // chunk 0 also clears the probe phase's counters and the statistics (no
    // probe starts before every chunk is done, chunk 0 included)
    if (bid == 0 && threadIdx.x == 0) {
        *b.tile_counter = 0u;
        *b.probe_done = 0u;
        *b.scatter_ready = 0u;
        if (b.stats) {
            b.stats[0] = b.stats[1] = b.stats[2] = b.stats[3] = b.stats[6] = 0ull;
            b.stats[5] = ~0ull;
        }
    }
    // this chunk is done once every thread's writes are visible: it counts
    // itself in sync->packed, which the probe phase waits for
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) red_release_add(&sync->packed, 1u);
    __syncthreads();  // sm is reused by the next chunk
}

// Bounded wait, by one thread, until every pack chunk of the batch is done;
// then the CTA may read the batch's records.
__device__ __forceinline__ void wait_packed(const PackSync *sync, uint32_t npack, uint32_t *err, uint32_t spin) {
    wait_eq(&sync->packed, npack, err, spin, 512u);
}

// The batch's error bits to the host word the batch names (the device word is
// cleared for the next batch); nothing when it names none.
__device__ __forceinline__ void hand_over_flags(const BatchView &b) {
    if (!b.err_out) return;
    *(volatile uint32_t *)b.err_out = atomicExch(b.err, 0u);
    __threadfence_system();
}

// Scatter phase, run by every CTA once its warps have left the probe loop.
// CTAs take chunks of 512 tiles by ticket; a chunk owner first acquires the
// count of probed tiles (all tiles done: their counts and first-tile marks,
// written by other CTAs), then scans the chunk's survivor counts, finds its
// base by a decoupled look-back over the chunks (replaces cudppScan,
// ParaPFD_Intersection.cu:262), writes the offsets of the queries whose first
// tile is in the chunk (replaces ucntResult, :301) and each tile's output
// position, and counts the chunk ready. Every CTA then copies survivors to
// the result array (replaces saCompact, :279) once all chunks are ready.
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
    if (nch == 0) {  // no tiles in the batch: every offset is 0
        for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q <= nq; q += gridDim.x * blockDim.x) offsets[q] = 0u;
        return;
    }
    for (;;) {
        // a chunk owner starts once every tile of the batch is probed (the
        // tiles' counts, slots and marks, written by other CTAs, are read
        // below); a CTA without a chunk reads nothing and leaves at once
        if (threadIdx.x == 0) {
            sm.c = atomicAdd(&sync->sticket, 1u);
            if (sm.c < nch) wait_eq(b.probe_done, T, b.err, spin, 128u);  // chunk owners only: few pollers
        }
        __syncthreads();
        const uint32_t c = sm.c;
        if (c >= nch) break;
        // the chunk's tiles: counts and first-tile marks (query + 1 for a
        // query's first tile, else 0), all loads in flight at once
        const uint32_t t0 = c * kSSChunk;
        const uint32_t ja = threadIdx.x * kPer, ta = t0 + ja;
        const uint32_t c0 = ta < T ? b.tile_count[ta] : 0u;
        const uint32_t c1 = ta + 1 < T ? b.tile_count[ta + 1] : 0u;
        const uint32_t f0 = ta < T ? b.tile_q[ta] : 0u;
        const uint32_t f1 = ta + 1 < T ? b.tile_q[ta + 1] : 0u;
        // a query before a first tile that has no tiles itself shares its offset
        const uint32_t pe0 = f0 > 1u ? b.tile_prefix[f0 - 2u] : 0xffffffffu;
        const uint32_t pe1 = f1 > 1u ? b.tile_prefix[f1 - 2u] : 0xffffffffu;
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
                    uint64_t sv = ld_acquire64(&chunk_state[idx]);
                    uint32_t spins = 0;
                    while ((uint32_t)(sv >> 34) != tag) {
                        if (++spins > spin) {
                            atomicOr(b.err, kErrScanSpin);
                            sv = chunk_word(tag, kPrefix, 0u);
                            break;
                        }
                        __nanosleep(32);
                        sv = ld_acquire64(&chunk_state[idx]);
                    }
                    st = (uint32_t)(sv >> 32) & 3u;
                    v = (uint32_t)sv;
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
            if (lane == 0) {
                sm.base = excl;
                st_release64(&chunk_state[c], chunk_word(tag, kPrefix, excl + tot));
            }
        }
        __syncthreads();
        const uint32_t base = sm.base;
        if (c == nch - 1 && threadIdx.x == 0 && (uint64_t)base + tot > cap) atomicOr(b.err, kErrCapacity);
        // offsets of the queries that start here (and of empty queries before them)
        if (f0) {
            offsets[f0 - 1u] = base + ex;
            if (pe0 == ta)
                for (uint32_t q = f0 - 1u; q > 0 && b.tile_prefix[q - 1u] == ta; --q) offsets[q - 1u] = base + ex;
        }
        if (f1) {
            offsets[f1 - 1u] = base + ex + c0;
            if (pe1 == ta + 1)
                for (uint32_t q = f1 - 1u; q > 0 && b.tile_prefix[q - 1u] == ta + 1; --q) offsets[q - 1u] = base + ex + c0;
        }
        if (c == nch - 1 && threadIdx.x == 0) {
            // the batch total, and the queries after the last tile (no tiles)
            offsets[nq] = base + tot;
            for (uint32_t q = nq; q > 0 && b.tile_prefix[q - 1u] >= T; --q) offsets[q - 1u] = base + tot;
        }
        // each tile's output position, in place of its first-tile mark (read above)
        if (ta < T) b.tile_q[ta] = base + ex;
        if (ta + 1 < T) b.tile_q[ta + 1] = base + ex + c0;
        // the chunk is ready once every thread's writes are visible
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) red_release_add(b.scatter_ready, 1u);
    }
    // Survivors, copied by every warp of the grid once every chunk is ready
    // (one acquire per CTA; the ready chunks' owners acquired the probed count
    // before reading the tiles, so the tiles' results are visible too). A
    // batch's survivors gather in the chunks of its heaviest queries, so the
    // copy is spread over the whole grid: warp w takes tiles w, w + nw, ...;
    // lane j fetches the count, slot and output position of the warp's j-th
    // tile of a round, all lanes at once, and the warp then copies the round's
    // non-empty tiles with eight independent loads per lane.
    if (threadIdx.x == 0) wait_eq(b.scatter_ready, nch, b.err, spin, 512u);
    __syncthreads();
    const uint32_t gw = blockIdx.x * (blockDim.x / 32) + w, nw = gridDim.x * (blockDim.x / 32);
    const uint32_t *__restrict__ scr = b.scratch;
    for (uint64_t j0 = 0; gw + j0 * nw < T; j0 += 32) {
        const uint64_t tt = gw + (j0 + lane) * nw;
        const uint32_t t = tt < T ? (uint32_t)tt : T;
        const uint32_t n = t < T ? b.tile_count[t] : 0u;
        const uint32_t o = n ? b.tile_q[t] : 0u, slot = n ? b.tile_slot[t] : 0u;
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
