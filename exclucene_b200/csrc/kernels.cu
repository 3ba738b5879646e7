// sm_100a kernels of the batched decode + AND-intersection path.
//
//   (whole-list decode, K1/K2, is in decode.cu)
//   k_pack           per-query term sort by list length + tiles of the
//                    shortest list (replaces CPUPreprocess, ParaPFD_Intersection.cu:126-227).
//   k_scan_excl      device-wide exclusive scan, single pass with decoupled
//                    look-back and bounded waits (replaces cudppScan).
//   k_probe<ALGO>    persistent kernel: each warp takes (query, tile) work
//                    items from an atomic queue, decodes the tile of the
//                    shortest list into smem, probes every longer list and
//                    compacts survivors with ballot/popc (replaces the search
//                    kernels, e.g. ParaPFD_Intersection_kernel.cu:145-458).
//   k_scatter        moves each tile's survivors to its scanned position and
//                    writes per-query offsets (replaces saCompact + ucntResult,
//                    ParaPFD_Intersection_kernel.cu:461-565).
#include <cstdio>

#include "excl_device.cuh"
#include "kernels.h"

namespace excl {

// ---------------------------------------------------------------------------
// Query pack: sort each query's terms by list length (stable insertion sort,
// ParaPFD_Intersection.cu:155-173) and count the tiles of its shortest list.

__global__ void k_pack(const ListDesc *__restrict__ lists, uint32_t nlists, const uint32_t *__restrict__ terms,
                       const uint32_t *__restrict__ toff, uint32_t nq, uint32_t *__restrict__ qterms,
                       uint32_t *__restrict__ qnterms, uint32_t *__restrict__ ntiles, uint32_t *__restrict__ nkeys,
                       uint32_t *__restrict__ tile_counter, uint32_t *__restrict__ err) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q == 0) *tile_counter = 0u;
    if (q >= nq) return;
    const uint32_t t0 = toff[q], t1 = toff[q + 1];
    uint32_t k = t1 >= t0 ? t1 - t0 : 0u;
    if (k > kMaxTerms) {
        atomicOr(err, kErrTerms);
        k = 0;
    }
    uint32_t id[kMaxTerms], len[kMaxTerms];
    for (uint32_t i = 0; i < k; ++i) {
        const uint32_t tid = terms[t0 + i];
        if (tid >= nlists) {
            atomicOr(err, kErrTermId);
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
    uint32_t *dst = qterms + (size_t)q * kMaxTerms;
    for (uint32_t i = 0; i < k; ++i) dst[i] = id[i];
    qnterms[q] = k;
    ntiles[q] = k ? lists[id[0]].ntiles : 0u;
    nkeys[q] = k ? len[0] : 0u;
}

// ---------------------------------------------------------------------------
// Exclusive scan (u32) with decoupled look-back. Block order comes from an
// atomic ticket, so a block only ever waits on blocks that are already running;
// every wait is bounded and raises kErrScanSpin when it gives up.

constexpr int kScanThreads = 256, kScanItems = 8, kScanTile = kScanThreads * kScanItems;
constexpr uint64_t kFlagA = 1ull << 32, kFlagP = 2ull << 32;
constexpr uint32_t kSpinLimit = 1u << 20;

__device__ __forceinline__ uint64_t ld_volatile(const uint64_t *p) { return *(const volatile uint64_t *)p; }
__device__ __forceinline__ void st_volatile(uint64_t *p, uint64_t v) { *(volatile uint64_t *)p = v; }

__global__ void __launch_bounds__(kScanThreads) k_scan_excl(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                            const uint32_t *__restrict__ n_dev, uint32_t n_host,
                                                            uint32_t n_max, uint64_t *__restrict__ state,
                                                            uint32_t *__restrict__ ticket, uint32_t *__restrict__ err) {
    __shared__ uint32_t s_bid, s_prefix;
    __shared__ uint32_t s_warp[kScanThreads / 32];
    __shared__ uint32_t s_data[kScanTile];
    uint32_t n = n_dev ? *n_dev : n_host;
    if (n > n_max) {
        // a length read from the device beyond the buffers: scan what fits, flag it
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(err, kErrCapacity);
        n = n_max;
    }
    if (threadIdx.x == 0) s_bid = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t bid = s_bid;
    const uint64_t base = (uint64_t)bid * kScanTile;
    if (base >= n && bid != 0) return;
    // coalesced load into smem, then each thread takes 8 consecutive items
    for (uint32_t i = threadIdx.x; i < kScanTile; i += kScanThreads)
        s_data[i] = (base + i < n) ? in[base + i] : 0u;
    __syncthreads();
    uint32_t v[kScanItems], sum = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        v[j] = s_data[threadIdx.x * kScanItems + j];
        sum += v[j];
    }
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t wv = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
        uint32_t wi = wv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= (uint32_t)o) wi += t;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = wi - wv;  // exclusive per warp
        const uint32_t agg = __shfl_sync(0xffffffffu, wi, kScanThreads / 32 - 1);
        uint32_t prefix = 0;
        if (bid == 0) {
            if (lane == 0) {
                __threadfence();
                st_volatile(&state[0], kFlagP | agg);
            }
        } else {
            if (lane == 0) {
                __threadfence();
                st_volatile(&state[bid], kFlagA | agg);
            }
            int p = (int)bid - 1;
            bool done = false;
            uint32_t spins = 0;
            while (!done) {
                const int idx = p - (int)lane;
                uint64_t st = idx >= 0 ? ld_volatile(&state[idx]) : kFlagP;
                while (__any_sync(0xffffffffu, (st >> 32) == 0)) {
                    if (++spins > kSpinLimit) {
                        if (lane == 0) atomicOr(err, kErrScanSpin);
                        st = kFlagP;  // give up: treat as zero so the kernel ends
                    } else {
                        __nanosleep(64);
                        if ((st >> 32) == 0) st = ld_volatile(&state[idx]);
                    }
                }
                const uint32_t pmask = __ballot_sync(0xffffffffu, (st >> 32) == 2);
                uint32_t val = (uint32_t)st;
                if (pmask) {
                    const uint32_t f = __ffs(pmask) - 1;
                    if (lane > f) val = 0;
                    done = true;
                } else {
                    p -= 32;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
                prefix += val;
            }
            if (lane == 0) {
                __threadfence();
                st_volatile(&state[bid], kFlagP | (prefix + agg));
            }
        }
        if (lane == 0) s_prefix = prefix;
        // the block holding element n-1 (or block 0 for n == 0) writes the total
        if (lane == 0 && base + kScanTile >= n) out[n] = prefix + agg;
    }
    __syncthreads();
    uint32_t run = s_prefix + s_warp[wid] + (incl - sum);
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        s_data[threadIdx.x * kScanItems + j] = run;
        run += v[j];
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kScanTile; i += kScanThreads)
        if (base + i < n) out[base + i] = s_data[i];
}

// ---------------------------------------------------------------------------
// Probe of one key against one longer list.

__device__ __forceinline__ int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }
__device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

template <int ALGO>
__device__ __forceinline__ bool probe_key(const DevIndexView &ix, const ListDesc &L, uint32_t key, uint32_t &fallback) {
    if (key < L.first_doc || key > L.last_doc) return false;
    uint32_t lo, hi;
    int64_t plo = 0, phi = -1;  // learned rank window (inclusive), when used
    bool learned = false;
    if ((ALGO == EXCL_ALGO_LEARNED || ALGO == EXCL_ALGO_AUTO) && L.model != kNoModel) {
        const ModelHdr m = ix.models.hdr[L.model];
        const float x = model_norm(m, key);
        const Leaf lf = ix.models.leaves[m.leaf_base + model_route(ix.models.grid, ix.models.bnd, m, key)];
        // no posting of the list routes to an empty leaf, and routing is deterministic
        if (lf.ehi < lf.elo) return false;
        if ((uint32_t)(lf.ehi - lf.elo) <= m.max_window) {
            const int pr = model_pred_rank(lf, x);
            plo = imax64(0, (int64_t)pr + lf.elo);
            phi = imin64((int64_t)L.n - 1, (int64_t)pr + lf.ehi);
            if (plo > phi) return false;
            learned = true;
        } else {
            ++fallback;
        }
    }
    if (learned) {
        lo = (uint32_t)(plo >> L.log2_block);
        hi = (uint32_t)(phi >> L.log2_block) + 1u;
    } else if (ALGO == EXCL_ALGO_BSEARCH) {
        lo = 0;
        hi = L.nseg;
    } else {
        const uint32_t b = (uint32_t)((uint64_t)key >> L.dir_shift);
        const uint32_t d0 = ldg(ix.dir + L.dir_base + b), d1 = ldg(ix.dir + L.dir_base + b + 1);
        lo = codec_is_hs(L.codec) ? d0 : (d0 ? d0 - 1u : 0u);
        hi = d1;
    }
    const int s = last_head_le(ix.seg_head + L.seg_base, lo, hi, key);
    if (s < (int)lo) return false;
    const uint32_t sg = L.seg_base + (uint32_t)s;
    const SegRec rec = ix.seg_rec[sg];
    const uint32_t *blk = ix.words + L.word_base + rec.off;
    if (codec_is_dgap(L.codec)) return dgap_find(blk, rec.count, ldg(ix.seg_head + sg), rec.aux, key);
    const BlkHdr h = blk_hdr(ldg(blk));
    const SegReg reg = ix.seg_reg[sg];
    const ResidParams rp = resid_params(L, rec, reg);
    int64_t t0 = 0, t1 = (int64_t)rec.count - 1;
    if (learned) {
        t0 = imax64(t0, plo - rec.start);
        t1 = imin64(t1, phi - rec.start);
    } else if (L.codec == EXCL_CODEC_SEGLRC || L.codec == EXCL_CODEC_HS_SEGLRC || L.codec == EXCL_CODEC_LRCSEG) {
        // Regression window (SegLRC_Intersection_kernel.cu:366-371): the pivot
        // (key - b) / a in IEEE single precision, widened by the fit's safe
        // range. The range was measured with this same expression on every
        // element, so a present key always lies inside.
        float a, bb;
        uint32_t rl, rr;
        int64_t off;
        if (L.codec == EXCL_CODEC_LRCSEG) {
            a = __uint_as_float(L.reg[0]);
            bb = __uint_as_float(L.reg[1]);
            rl = L.reg[2];
            rr = L.reg[3];
            off = rec.start;
        } else {
            a = reg.a;
            bb = reg.b;
            rl = reg.L;
            rr = reg.R;
            off = 0;
        }
        const float px = __fdiv_rn(__fsub_rn(__uint2float_rn(key), bb), a);
        if (isfinite(px) && fabsf(px) < 2.0e9f) {
            const int64_t P = (int64_t)__float2int_rz(px) - off;
            t0 = imax64(t0, P - (int64_t)rl);
            t1 = imin64(t1, P + (int64_t)rr);
        }
    }
    if (t0 > t1) return false;
    return resid_find(blk, h, rp, rec.count, (int)t0, (int)t1, key);
}

// ---------------------------------------------------------------------------
// Persistent probe kernel.

template <int ALGO, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_probe(DevIndexView ix, BatchView b) {
    __shared__ uint32_t s_keys[WARPS][kTileKeys];
    __shared__ ListDesc s_list[WARPS];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t *keys = s_keys[w];
    ListDesc &L = s_list[w];
    const uint32_t nq = b.nq;
    const uint32_t T = min(b.tile_prefix[nq], b.max_tiles);
    uint32_t probes = 0, fallbacks = 0, nkeys = 0;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(b.tile_counter, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= T) break;
        // query owning tile t: last q with tile_prefix[q] <= t
        uint32_t lo = 0, hi = nq;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (b.tile_prefix[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const uint32_t q = lo;
        const uint32_t ti = t - b.tile_prefix[q];
        const uint32_t k = b.qnterms[q];
        const uint32_t *qt = b.qterms + (size_t)q * kMaxTerms;
        __syncwarp();
        if (lane < 5) reinterpret_cast<uint4 *>(&L)[lane] = reinterpret_cast<const uint4 *>(ix.lists + qt[0])[lane];
        __syncwarp();
        // decode the tile's keys: one fixed segment, or 1..255 consecutive
        // variable segments / one 256-slice of a large segment
        uint32_t kc = 0, first_elem;
        if (L.log2_block) {
            const uint32_t sg = L.seg_base + ti;
            kc = ix.seg_rec[sg].count;
            first_elem = ti << L.log2_block;
            warp_decode(ix, L, sg, 0, kc, keys, lane);
        } else {
            const uint64_t tm = ix.tilemap[L.tile_base + ti];
            const uint32_t sg0 = L.seg_base + (uint32_t)(tm >> 32);
            const uint32_t e0 = (uint32_t)(tm >> 8) & kTileMaxE0, ns = (uint32_t)tm & 0xffu;
            first_elem = ix.seg_rec[sg0].start + e0;
            for (uint32_t g = 0; g < ns; ++g) {
                const uint32_t c = min(kTileKeys - kc, ix.seg_rec[sg0 + g].count - (g ? 0u : e0));
                warp_decode(ix, L, sg0 + g, g ? 0u : e0, c, keys + kc, lane);
                kc += c;
            }
        }
        nkeys += kc;
        uint32_t alive = kc;
        for (uint32_t j = 1; j < k && alive; ++j) {
            __syncwarp();
            if (lane < 5) reinterpret_cast<uint4 *>(&L)[lane] = reinterpret_cast<const uint4 *>(ix.lists + qt[j])[lane];
            __syncwarp();
            uint32_t nout = 0;
            for (uint32_t base = 0; base < alive; base += 32) {
                const uint32_t i = base + lane;
                const bool valid = i < alive;
                const uint32_t key = valid ? keys[i] : 0u;
                const bool f = valid && probe_key<ALGO>(ix, L, key, fallbacks);
                probes += valid;
                const uint32_t m = __ballot_sync(0xffffffffu, f);
                const uint32_t pos = nout + __popc(m & ((1u << lane) - 1u));
                __syncwarp();
                if (f) keys[pos] = key;
                nout += __popc(m);
            }
            __syncwarp();
            alive = nout;
        }
        // survivors go to the tile's key-indexed slot (its keys' positions in
        // the batch's concatenated shortest lists)
        const uint64_t slot = (uint64_t)b.key_base[q] + first_elem;
        if (slot + kc > b.max_keys) {
            if (lane == 0) atomicOr(b.err, kErrCapacity);
            alive = 0;
        }
        uint32_t *dst = b.scratch + slot;
        for (uint32_t i = lane; i < alive; i += 32) dst[i] = keys[i];
        if (lane == 0) {
            b.tile_count[t] = alive;
            b.tile_slot[t] = (uint32_t)slot;
        }
        __syncwarp();
    }
    if (b.stats) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            probes += __shfl_xor_sync(0xffffffffu, probes, o);
            fallbacks += __shfl_xor_sync(0xffffffffu, fallbacks, o);
        }
        if (lane == 0) {
            atomicAdd((unsigned long long *)&b.stats[0], (unsigned long long)probes);
            atomicAdd((unsigned long long *)&b.stats[1], (unsigned long long)fallbacks);
            atomicAdd((unsigned long long *)&b.stats[2], (unsigned long long)nkeys);
        }
    }
}

// ---------------------------------------------------------------------------
// Scatter survivors and write per-query offsets.

__global__ void k_scatter(BatchView b, const uint32_t *__restrict__ tile_out, uint32_t *__restrict__ offsets,
                          uint32_t *__restrict__ docids, uint64_t cap) {
    const uint32_t nq = b.nq;
    const uint32_t T = min(b.tile_prefix[nq], b.max_tiles);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0 && tile_out[T] > cap) atomicOr(b.err, kErrCapacity);
    for (uint32_t t = gw; t < T; t += nw) {
        const uint32_t c = b.tile_count[t];
        const uint64_t o = tile_out[t];
        const uint32_t *src = b.scratch + b.tile_slot[t];
        for (uint32_t i = lane; i < c; i += 32)
            if (o + i < cap) docids[o + i] = src[i];
    }
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t q = gt; q <= nq; q += gridDim.x * blockDim.x) offsets[q] = tile_out[min(b.tile_prefix[q], T)];
}

// ---------------------------------------------------------------------------
// Launchers.

int launch_pack(const ListDesc *lists, uint32_t nlists, const uint32_t *terms, const uint32_t *toff, uint32_t nq,
                const BatchView &b, uint32_t *ntiles, uint32_t *nkeys, cudaStream_t st) {
    const uint32_t blocks = std::max(1u, (nq + 127) / 128);
    k_pack<<<blocks, 128, 0, st>>>(lists, nlists, terms, toff, nq, const_cast<uint32_t *>(b.qterms),
                                    const_cast<uint32_t *>(b.qnterms), ntiles, nkeys, b.tile_counter, b.err);
    return (int)cudaGetLastError();
}

uint32_t scan_blocks_for(uint64_t n) { return (uint32_t)std::max<uint64_t>(1, (n + kScanTile - 1) / kScanTile); }

int launch_scan(const uint32_t *in, uint32_t *out, const uint32_t *n_dev, uint32_t n_host, uint64_t max_n,
                uint64_t *state, uint32_t *ticket, uint32_t *err, cudaStream_t st) {
    const uint32_t blocks = scan_blocks_for(max_n);
    cudaMemsetAsync(state, 0, sizeof(uint64_t) * blocks, st);
    cudaMemsetAsync(ticket, 0, sizeof(uint32_t), st);
    const uint32_t n_max = (uint32_t)std::min<uint64_t>(max_n, 0xffffffffull);
    k_scan_excl<<<blocks, kScanThreads, 0, st>>>(in, out, n_dev, n_host, n_max, state, ticket, err);
    return (int)cudaGetLastError();
}

template <int ALGO, int WARPS>
static void launch_probe_t(const DevIndexView &ix, const BatchView &b, uint32_t blocks, cudaStream_t st) {
    k_probe<ALGO, WARPS><<<blocks, WARPS * 32, 0, st>>>(ix, b);
}

template <int WARPS>
static void launch_probe_w(const DevIndexView &ix, const BatchView &b, int algo, uint32_t blocks, cudaStream_t st) {
    switch (algo) {
        case EXCL_ALGO_BSEARCH: launch_probe_t<EXCL_ALGO_BSEARCH, WARPS>(ix, b, blocks, st); break;
        case EXCL_ALGO_HASHSEG: launch_probe_t<EXCL_ALGO_HASHSEG, WARPS>(ix, b, blocks, st); break;
        case EXCL_ALGO_LEARNED: launch_probe_t<EXCL_ALGO_LEARNED, WARPS>(ix, b, blocks, st); break;
        default: launch_probe_t<EXCL_ALGO_AUTO, WARPS>(ix, b, blocks, st); break;
    }
}

int launch_probe(const DevIndexView &ix, const BatchView &b, int algo, int warps, int ctas_per_sm, int nsm,
                 cudaStream_t st) {
    const uint32_t blocks = (uint32_t)std::max(1, nsm * ctas_per_sm);
    switch (warps) {
        case 4: launch_probe_w<4>(ix, b, algo, blocks, st); break;
        case 16: launch_probe_w<16>(ix, b, algo, blocks, st); break;
        default: launch_probe_w<8>(ix, b, algo, blocks, st); break;
    }
    return (int)cudaGetLastError();
}

int launch_scatter(const BatchView &b, const uint32_t *tile_out, uint32_t *offsets, uint32_t *docids, uint64_t cap,
                   int nsm, cudaStream_t st) {
    k_scatter<<<nsm * 4, 256, 0, st>>>(b, tile_out, offsets, docids, cap);
    return (int)cudaGetLastError();
}

}  // namespace excl
