// The batch pipeline's bookkeeping kernels, fused so a batch is three launches
// (k_pack_scan -> k_probe -> k_scan_scatter) with no memsets in between.
//
//   k_pack_scan     per query: sort the terms by list length (stable insertion
//                   sort, ParaPFD_Intersection.cu:155-173), count the shortest
//                   list's tiles and docIDs; then the exclusive prefixes of both
//                   over the batch. The <= 256 CTAs publish their totals with
//                   release/acquire flags and each sums its predecessors'; the
//                   last CTA to finish clears the flags for the next batch.
//                   Also resets the probe's work counter and statistics.
//   k_scan_scatter  cooperative: per-chunk sums of the per-tile survivor
//                   counts, grid sync, chunk prefixes and per-tile output
//                   positions, survivors copied to the result array (replaces
//                   cudppScan + saCompact, ParaPFD_Intersection.cu:262,279),
//                   grid sync, per-query offsets (replaces ucntResult, :301).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "kernels.h"

namespace cg = cooperative_groups;

namespace excl {

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

constexpr uint32_t kSpin = 1u << 22;

// Block-wide exclusive scan of two values at once; returns the block totals.
__device__ __forceinline__ void block_scan2(uint32_t a, uint32_t b, uint32_t &ea, uint32_t &eb, uint32_t &ta,
                                            uint32_t &tb, uint32_t *sa, uint32_t *sb) {
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t ia = a, ib = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t xa = __shfl_up_sync(0xffffffffu, ia, o), xb = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= (uint32_t)o) {
            ia += xa;
            ib += xb;
        }
    }
    if (lane == 31) {
        sa[w] = ia;
        sb[w] = ib;
    }
    __syncthreads();
    if (w == 0) {
        uint32_t va = lane < nw ? sa[lane] : 0u, vb = lane < nw ? sb[lane] : 0u;
        uint32_t ja = va, jb = vb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t xa = __shfl_up_sync(0xffffffffu, ja, o), xb = __shfl_up_sync(0xffffffffu, jb, o);
            if (lane >= (uint32_t)o) {
                ja += xa;
                jb += xb;
            }
        }
        if (lane < nw) {
            sa[lane] = ja - va;
            sb[lane] = jb - vb;
        }
        if (lane == 31) {
            sa[32] = ja;
            sb[32] = jb;
        }
    }
    __syncthreads();
    ea = sa[w] + ia - a;
    eb = sb[w] + ib - b;
    ta = sa[32];
    tb = sb[32];
}

__global__ void __launch_bounds__(kPackThreads) k_pack_scan(const ListDesc *__restrict__ lists, uint32_t nlists,
                                                            const uint32_t *__restrict__ terms,
                                                            const uint32_t *__restrict__ toff, uint32_t nq,
                                                            BatchView b, PackSync *__restrict__ sync) {
    __shared__ uint32_t sa[33], sb[33], s_pre[2], s_et[kPackThreads];
    static_assert(kPackMaxCtas <= 32 * 8, "warp 0 reads up to 8 predecessors per lane");
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t nt = 0, nk = 0;
    if (q < nq) {
        const uint32_t t0 = toff[q], t1 = toff[q + 1];
        uint32_t k = t1 >= t0 ? t1 - t0 : 0u;
        if (k > kMaxTerms) {
            atomicOr(b.err, kErrTerms);
            k = 0;
        }
        uint32_t id[kMaxTerms], len[kMaxTerms];
        for (uint32_t i = 0; i < k; ++i) {
            const uint32_t tid = terms[t0 + i];
            if (tid >= nlists) {
                atomicOr(b.err, kErrTermId);
                k = 0;
                break;
            }
            id[i] = tid;
            len[i] = lists[tid].n;
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
        uint32_t *dst = const_cast<uint32_t *>(b.qterms) + (size_t)q * kMaxTerms;
        for (uint32_t i = 0; i < k; ++i) dst[i] = id[i];
        const_cast<uint32_t *>(b.qnterms)[q] = k;
        nt = k ? lists[id[0]].ntiles : 0u;
        nk = k ? len[0] : 0u;
    }
    uint32_t et, ek, bt, bk;
    block_scan2(nt, nk, et, ek, bt, bk, sa, sb);
    const uint32_t bid = blockIdx.x;
    if (threadIdx.x == 0) {
        sync->agg_t[bid] = bt;
        sync->agg_k[bid] = bk;
        st_release(&sync->flag[bid], 1u);
    }
    if (threadIdx.x < 32) {
        // warp 0: the predecessors' totals, read in parallel (all CTAs are resident)
        const uint32_t lane = threadIdx.x;
        uint32_t pt = 0, pk = 0;
        for (uint32_t p = lane; p < bid; p += 32) {
            uint32_t spins = 0;
            while (ld_acquire(&sync->flag[p]) == 0u) {
                if (++spins > kSpin) {
                    atomicOr(b.err, kErrScanSpin);
                    break;
                }
                __nanosleep(32);
            }
            pt += sync->agg_t[p];
            pk += sync->agg_k[p];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            pt += __shfl_xor_sync(0xffffffffu, pt, o);
            pk += __shfl_xor_sync(0xffffffffu, pk, o);
        }
        if (lane == 0) {
            s_pre[0] = pt;
            s_pre[1] = pk;
        }
    }
    if (threadIdx.x == 0) {
        const uint32_t pt = s_pre[0], pk = s_pre[1];
        if (bid == gridDim.x - 1) {
            const_cast<uint32_t *>(b.tile_prefix)[nq] = pt + bt;
            const_cast<uint32_t *>(b.key_base)[nq] = pk + bk;
            if ((uint64_t)pt + bt > b.max_tiles || (uint64_t)pk + bk > b.max_keys) atomicOr(b.err, kErrCapacity);
        }
        if (bid == 0) {
            *b.tile_counter = 0u;
            if (b.stats) b.stats[0] = b.stats[1] = b.stats[2] = 0ull;
        }
        // the last CTA to get here clears the flags for the next batch
        __threadfence();
        if (atomicAdd(&sync->done, 1u) == gridDim.x - 1) {
            for (uint32_t p = 0; p < gridDim.x; ++p) sync->flag[p] = 0u;
            sync->done = 0u;
            __threadfence();
        }
    }
    s_et[threadIdx.x] = et;
    __syncthreads();
    const uint32_t pt = s_pre[0];
    if (q < nq) {
        const_cast<uint32_t *>(b.tile_prefix)[q] = pt + et;
        const_cast<uint32_t *>(b.key_base)[q] = s_pre[1] + ek;
    }
    // owner of each of this CTA's tiles: the last query whose first tile is
    // at or before it (queries with no tiles share their successor's start)
    for (uint32_t tl = threadIdx.x; tl < bt && pt + tl < b.max_tiles; tl += blockDim.x) {
        uint32_t lo = 0, hi = blockDim.x - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (s_et[mid] <= tl) lo = mid;
            else hi = mid - 1;
        }
        b.tile_q[pt + tl] = blockIdx.x * blockDim.x + lo;
    }
}

__global__ void __launch_bounds__(kSSThreads) k_scan_scatter(BatchView b, uint32_t *__restrict__ tile_out,
                                                             uint32_t *__restrict__ chunk_agg,
                                                             uint32_t *__restrict__ offsets,
                                                             uint32_t *__restrict__ docids, uint64_t cap) {
    cg::grid_group grid = cg::this_grid();
    __shared__ uint32_t s_red[kSSThreads / 32 + 1];
    __shared__ uint32_t sa[33], sb[33];
    constexpr int kPer = kSSChunk / kSSThreads;  // tiles per thread in a chunk
    const uint32_t nq = b.nq;
    const uint32_t T = min(b.tile_prefix[nq], b.max_tiles);
    const uint32_t nch = (T + kSSChunk - 1) / kSSChunk;
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    // phase 1: survivors per chunk of tiles
    for (uint32_t c = blockIdx.x; c < nch; c += gridDim.x) {
        uint32_t s = 0;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const uint32_t t = c * kSSChunk + j * kSSThreads + threadIdx.x;
            if (t < T) s += b.tile_count[t];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) s_red[w] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t tot = 0;
            for (int i = 0; i < kSSThreads / 32; ++i) tot += s_red[i];
            chunk_agg[c] = tot;
        }
        __syncthreads();
    }
    grid.sync();
    // phase 2: output position of every tile (chunk prefix + scan inside the chunk)
    for (uint32_t c = blockIdx.x; c < nch; c += gridDim.x) {
        uint32_t pre = 0;
        for (uint32_t i = threadIdx.x; i < c; i += kSSThreads) pre += chunk_agg[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) pre += __shfl_xor_sync(0xffffffffu, pre, o);
        if (lane == 0) s_red[w] = pre;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t tot = 0;
            for (int i = 0; i < kSSThreads / 32; ++i) tot += s_red[i];
            s_red[kSSThreads / 32] = tot;
        }
        __syncthreads();
        const uint32_t base = s_red[kSSThreads / 32];
        uint32_t cnt[kPer], sum = 0;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const uint32_t t = c * kSSChunk + threadIdx.x * kPer + j;
            cnt[j] = t < T ? b.tile_count[t] : 0u;
            sum += cnt[j];
        }
        uint32_t ex, e2, tot, t2;
        block_scan2(sum, 0u, ex, e2, tot, t2, sa, sb);
        uint32_t run = base + ex;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const uint32_t t = c * kSSChunk + threadIdx.x * kPer + j;
            if (t < T) tile_out[t] = run;
            run += cnt[j];
        }
        if (c == nch - 1 && threadIdx.x == kSSThreads - 1) tile_out[T] = run;
        __syncthreads();
    }
    if (nch == 0 && blockIdx.x == 0 && threadIdx.x == 0) tile_out[0] = 0u;
    grid.sync();
    // phase 3: every warp of the grid moves survivors; then the query offsets
    if (blockIdx.x == 0 && threadIdx.x == 0 && tile_out[T] > cap) atomicOr(b.err, kErrCapacity);
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = gw; t < T; t += nw) {
        const uint32_t n = b.tile_count[t];
        if (n == 0) continue;
        const uint64_t o = tile_out[t];
        const uint32_t *src = b.scratch + b.tile_slot[t];
        for (uint32_t k = lane; k < n; k += 32)
            if (o + k < cap) docids[o + k] = src[k];
    }
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t q = gt; q <= nq; q += gridDim.x * blockDim.x) offsets[q] = tile_out[min(b.tile_prefix[q], T)];
}

int launch_pack_scan(const ListDesc *lists, uint32_t nlists, const uint32_t *terms, const uint32_t *toff, uint32_t nq,
                     const BatchView &b, PackSync *sync, cudaStream_t st) {
    if (nq > kPackMaxQueries) return (int)cudaErrorInvalidValue;
    const uint32_t blocks = std::max(1u, (nq + kPackThreads - 1) / kPackThreads);
    k_pack_scan<<<blocks, kPackThreads, 0, st>>>(lists, nlists, terms, toff, nq, b, sync);
    return (int)cudaGetLastError();
}

int scan_scatter_grid(int nsm) {
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && cached[dev]) return cached[dev];
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scan_scatter, kSSThreads, 0);
    const int g = std::max(1, std::min(per_sm, 1) * nsm);
    if (dev >= 0 && dev < 64) cached[dev] = g;
    return g;
}

int launch_scan_scatter(const BatchView &b, uint32_t *tile_out, uint32_t *chunk_agg, uint32_t *offsets,
                        uint32_t *docids, uint64_t cap, int nsm, cudaStream_t st) {
    const int grid = scan_scatter_grid(nsm);
    BatchView bb = b;
    void *args[] = {&bb, &tile_out, &chunk_agg, &offsets, &docids, &cap};
    return (int)cudaLaunchCooperativeKernel((const void *)k_scan_scatter, dim3(grid), dim3(kSSThreads), args, 0, st);
}

}  // namespace excl
