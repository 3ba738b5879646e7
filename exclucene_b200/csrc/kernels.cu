// sm_100a kernels of the batched AND-intersection path: the probe kernel
// and the per-key search it runs against each longer list. The batch's
// bookkeeping kernels (query pack + prefixes, survivor scatter) are in
// pipeline.cu; whole-list decode is in decode.cu.
//
//   k_probe<ALGO>    persistent kernel: each warp takes (query, tile) work
//                    items from an atomic queue, decodes the tile of the
//                    shortest list into smem, probes every longer list and
//                    compacts survivors with ballot/popc (replaces the search
//                    kernels, e.g. ParaPFD_Intersection_kernel.cu:145-458).
#include <cstdio>

#include "excl_device.cuh"
#include "kernels.h"

namespace excl {

// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }
__device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

// Probe of K keys of one lane against one longer list L. Each key walks a
// chain of dependent loads: directory bucket (or learned model, or a binary
// search over all heads) -> segment heads -> segment record (head, block
// offset, count, base/median, descriptor, segment regression) -> block words
// (a d-gap walk from the head or median, ParaPFD_Intersection_kernel.cu:
// 383-447, or a binary search over random-access residuals inside the
// regression window, SegLRC_Intersection_kernel.cu:366-393). Every stage
// issues the loads of all K keys before using any, so K > 1 keeps K chains
// in flight per lane. Bit k of `act`: key[k] is valid; bit k of the result:
// key[k] is in L.
template <int ALGO, int KIND, int K>
__device__ __forceinline__ uint32_t probe_keys(const DevIndexView &ix, const ListDesc &L, const uint32_t (&key)[K],
                                               uint32_t act, uint32_t &fallback) {
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (key[k] < L.first_doc || key[k] > L.last_doc) act &= ~(1u << k);
    if (!act) return 0u;
    uint32_t lo[K] = {}, hi[K] = {};
    uint32_t plo[K] = {}, phi[K] = {};  // learned rank window (inclusive, within the list)
    uint32_t lrn = 0;                   // bit k: key k is searched in its learned window
    if ((ALGO == EXCL_ALGO_LEARNED || ALGO == EXCL_ALGO_AUTO) && L.model != kNoModel) {
        const ModelHdr m = ix.models.hdr[L.model];
        const uint32_t *bd = ix.models.bnd + m.bnd_base;
        // routing (model_route): the grid cell bounds the leaf, the leaf
        // boundaries resolve it (last l in [lo, hi] with bnd[l] <= key)
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (act >> k & 1u) {
                const uint32_t j = (key[k] - m.first) >> m.grid_shift;
                lo[k] = ix.models.grid[m.grid_base + j];
                hi[k] = ix.models.grid[m.grid_base + j + 1];
            }
        for (;;) {
            uint32_t more = 0;
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (lo[k] < hi[k]) {
                    const uint32_t mid = (lo[k] + hi[k] + 1) >> 1;
                    if (__ldg(bd + mid) <= key[k]) lo[k] = mid;
                    else hi[k] = mid - 1;
                    more |= lo[k] < hi[k];
                }
            if (!more) break;
        }
        Leaf lf[K];
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (act >> k & 1u) lf[k] = ix.models.leaves[m.leaf_base + lo[k]];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!(act >> k & 1u)) continue;
            // no posting of the list routes to an empty leaf, and routing is deterministic
            if (lf[k].ehi < lf[k].elo) {
                act &= ~(1u << k);
            } else if ((uint32_t)(lf[k].ehi - lf[k].elo) <= m.max_window) {
                const int pr = model_pred_rank(lf[k], model_norm(m, key[k]));
                const int64_t wl = imax64(0, (int64_t)pr + lf[k].elo);
                const int64_t wh = imin64((int64_t)L.n - 1, (int64_t)pr + lf[k].ehi);
                if (wl > wh) {
                    act &= ~(1u << k);
                } else {
                    lrn |= 1u << k;
                    plo[k] = (uint32_t)wl;
                    phi[k] = (uint32_t)wh;
                    lo[k] = plo[k] >> L.log2_block;
                    hi[k] = (phi[k] >> L.log2_block) + 1u;
                }
            } else {
                ++fallback;
            }
        }
    }
    // segment: the last one whose head is <= key. s[k] is the best segment
    // known so far (a head <= key), bit k of `hit` says it is one; [lo, hi)
    // holds the candidates after it. Learned windows and BSEARCH start with
    // no known segment; a directory entry carries the head of its segment,
    // so the bucket's first candidate is settled by the directory load.
    int s[K];
    uint32_t hit = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        s[k] = (int)lo[k] - 1;
        if (!(act >> k & 1u)) {
            lo[k] = hi[k] = 0;
        } else if (!(lrn >> k & 1u)) {
            if (ALGO == EXCL_ALGO_BSEARCH) {
                lo[k] = 0;
                hi[k] = L.nseg;
                s[k] = -1;
            } else {
                const uint32_t b = (uint32_t)((uint64_t)key[k] >> L.dir_shift);
                const uint2 e0 = ix.dir[L.dir_base + b], e1 = ix.dir[L.dir_base + b + 1];
                // fixed blocks: the segment before the bucket's first may hold
                // the key (it starts in an earlier bucket, so its head < key);
                // HS: only the bucket's own segments
                hi[k] = e1.x;
                if (e0.x < e1.x && e0.y <= key[k]) {
                    s[k] = (int)e0.x;
                    lo[k] = e0.x + 1u;
                    hit |= 1u << k;
                } else {
                    s[k] = (int)e0.x - 1;
                    lo[k] = hi[k];
                    if (!codec_is_hs(L.codec) && e0.x > 0) hit |= 1u << k;
                }
            }
        }
    }
    // Binary search over the remaining candidates (the dense heads for
    // BSEARCH, the records' heads otherwise) down to at most four, whose heads
    // are then loaded at once.
    const ProbeRec *prs = ix.seg_probe + L.seg_base;
    const uint32_t *hb = ALGO == EXCL_ALGO_BSEARCH ? ix.seg_head + L.seg_base : &prs[0].head;
    constexpr uint32_t hs = ALGO == EXCL_ALGO_BSEARCH ? 1u : (uint32_t)(sizeof(ProbeRec) / 4);
    for (;;) {
        uint32_t more = 0;
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (hi[k] > lo[k] + 4u) {
                const uint32_t mid = (lo[k] + hi[k]) >> 1;
                if (ldg(hb + (size_t)mid * hs) <= key[k]) {
                    lo[k] = mid + 1;
                    s[k] = (int)mid;
                    hit |= 1u << k;
                } else {
                    hi[k] = mid;
                }
                more |= hi[k] > lo[k] + 4u;
            }
        if (!more) break;
    }
    // one candidate and none before it (a learned window inside one segment):
    // its head is checked from its record instead of loaded first
    uint32_t one = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (hi[k] == lo[k] + 1u && !(hit >> k & 1u)) {
            s[k] = (int)lo[k];
            one |= 1u << k;
            continue;
        }
        uint32_t h4[4];
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) h4[j] = lo[k] + j < hi[k] ? ldg(hb + (size_t)(lo[k] + j) * hs) : 0xffffffffu;
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j)
            if (lo[k] + j < hi[k] && h4[j] <= key[k]) {
                s[k] = (int)(lo[k] + j);
                hit |= 1u << k;
            }
    }
    act &= hit | one;
    if (!act) return 0u;
    // segment records: head, block offset, aux, count | descriptor, regression
    uint4 q0[K], q1[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (act >> k & 1u) {
            q0[k] = __ldg(reinterpret_cast<const uint4 *>(prs + s[k]));
            q1[k] = __ldg(reinterpret_cast<const uint4 *>(prs + s[k]) + 1);
        }
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((act & one) >> k & 1u && key[k] < q0[k].x) act &= ~(1u << k);
    if (!act) return 0u;
    const uint32_t *lw = ix.words + L.word_base;
    uint32_t found = 0;
    if (KIND == kKindDgap || (KIND == kKindAny && codec_is_dgap(L.codec))) {
        // d-gap walks: each is a stream over one block
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (act >> k & 1u) {
                const uint32_t *blk = lw + q0[k].y;
                const BlkHdr h = blk_hdr(q1[k].x);
                const bool f = (KIND == kKindAny && codec_is_newpfd(L.codec))
                                   ? dgap_find_newpfd(blk, h, q0[k].w, q0[k].x, q0[k].z, key[k])
                                   : dgap_find(blk, h, q0[k].w, q0[k].x, q0[k].z, key[k]);
                found |= (uint32_t)f << k;
            }
        return found;
    }
    if constexpr (KIND != kKindDgap) {
        // residual codecs: windows, then one binary search step of every key per round
        int t0[K], t1[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            t0[k] = 0;
            t1[k] = -1;
            if (!(act >> k & 1u)) continue;
            // list position of the segment: only learned windows and the
            // LRC/LRCSeg predictors use it, and those lists have fixed blocks
            const uint32_t start = (uint32_t)s[k] << L.log2_block, count = q0[k].w;
            int64_t w0 = 0, w1 = (int64_t)count - 1;
            if (lrn >> k & 1u) {
                w0 = imax64(w0, (int64_t)plo[k] - start);
                w1 = imin64(w1, (int64_t)phi[k] - start);
            } else if (L.codec == EXCL_CODEC_SEGLRC || L.codec == EXCL_CODEC_HS_SEGLRC || L.codec == EXCL_CODEC_LRCSEG) {
                // Regression window (SegLRC_Intersection_kernel.cu:366-371): the
                // pivot (key - b) / a in IEEE single precision, widened by the
                // fit's safe range. The range was measured with this same
                // expression on every element, so a present key always lies inside.
                float a, bb;
                uint32_t rl, rr;
                int64_t off;
                if (L.codec == EXCL_CODEC_LRCSEG) {
                    a = __uint_as_float(L.reg[0]);
                    bb = __uint_as_float(L.reg[1]);
                    rl = L.reg[2];
                    rr = L.reg[3];
                    off = start;
                } else {
                    a = __uint_as_float(q1[k].y);
                    bb = __uint_as_float(q1[k].z);
                    rl = (q1[k].w & 0xffffu) == kProbeUnbounded ? 0x7fffffffu : (q1[k].w & 0xffffu);
                    rr = (q1[k].w >> 16) == kProbeUnbounded ? 0x7fffffffu : (q1[k].w >> 16);
                    off = 0;
                }
                const float px = __fdiv_rn(__fsub_rn(__uint2float_rn(key[k]), bb), a);
                if (isfinite(px) && fabsf(px) < 2.0e9f) {
                    const int64_t P = (int64_t)__float2int_rz(px) - off;
                    w0 = imax64(w0, P - (int64_t)rl);
                    w1 = imin64(w1, P + (int64_t)rr);
                }
            }
            if (w0 <= w1) {
                t0[k] = (int)w0;
                t1[k] = (int)w1;
            }
        }
        for (;;) {
            uint32_t more = 0;
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (t0[k] <= t1[k]) {
                    const int mid = (t0[k] + t1[k]) >> 1;
                    SegRec rec;
                    rec.start = (uint32_t)s[k] << L.log2_block;
                    rec.aux = q0[k].z;
                    SegReg reg;
                    reg.a = __uint_as_float(q1[k].y);
                    reg.b = __uint_as_float(q1[k].z);
                    const ResidParams rp = resid_params(L, rec, reg);
                    const BlkHdr h = blk_hdr(q1[k].x);
                    const uint32_t v =
                        resid_value(rp, (uint32_t)mid, block_value_ra(lw + q0[k].y, h, q0[k].w, (uint32_t)mid));
                    if (v == key[k]) {
                        found |= 1u << k;
                        t1[k] = t0[k] - 1;
                    } else if (v < key[k]) {
                        t0[k] = mid + 1;
                    } else {
                        t1[k] = mid - 1;
                    }
                    more |= t0[k] <= t1[k];
                }
            if (!more) break;
        }
    }
    return found;
}

// Segment of L (list-relative) whose head is the last one <= key, found with
// the directory (or a binary search over all heads for BSEARCH); -1 if key
// precedes the list.
template <int ALGO>
__device__ __forceinline__ int locate_segment(const DevIndexView &ix, const ListDesc &L, uint32_t key) {
    if (key < L.first_doc) return -1;
    if (key > L.last_doc) return (int)L.nseg - 1;
    uint32_t lo = 0, hi = L.nseg;
    if (ALGO != EXCL_ALGO_BSEARCH) {
        const uint32_t bk = (uint32_t)((uint64_t)key >> L.dir_shift);
        const uint32_t d0 = ix.dir[L.dir_base + bk].x, d1 = ix.dir[L.dir_base + bk + 1].x;
        lo = codec_is_hs(L.codec) ? d0 : (d0 ? d0 - 1u : 0u);
        hi = d1;
    }
    return last_head_le(ix.seg_head + L.seg_base, lo, hi, key);
}

// ---------------------------------------------------------------------------
// Persistent probe kernel.
//
// For each longer list a tile chooses between two methods (the merge-path /
// probe choice): when the tile's surviving keys span few of the list's
// segments (at most b.merge_segs, whose docIDs fit kMergeCap), the warp
// decodes that span into shared memory once and every key is looked up there;
// otherwise each key is probed on its own (probe_keys).

// MINB: resident 8-warp CTAs per SM the register budget is cut for (4: 64
// registers; 5: 48; 6: 40), traded for more probes in flight; the launch
// shape is an autotuner choice. KIND: the codec family the instance handles
// (kKindAny for mixed indexes); a one-family instance needs fewer registers
// (residual codecs: no spills at 64, the 64-register spills at 48).
template <int ALGO, int WARPS, int MINB, int KIND>
__global__ void __launch_bounds__(WARPS * 32, (8 / WARPS) * MINB) k_probe(DevIndexView ix, BatchView b) {
    __shared__ uint32_t s_keys[WARPS][kTileKeys];
    __shared__ uint32_t s_merge[WARPS][kMergeCap];
    __shared__ ListDesc s_list[WARPS];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t *keys = s_keys[w];  // the tile's keys (a sub-range of the decoded segment when tiles are cut)
    uint32_t *mbuf = s_merge[w];
    ListDesc &L = s_list[w];
    const uint32_t T = min(b.tile_prefix[b.nq], b.max_tiles);
    uint32_t probes = 0, fallbacks = 0, nkeys = 0, merges = 0;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(b.tile_counter, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= T) break;
        const uint32_t q = b.tile_q[t];  // owner written by the pack kernel
        const uint32_t ti = t - b.tile_prefix[q];
        const uint32_t k = b.qnterms[q];
        const uint32_t *qt = b.qterms + (size_t)q * kMaxTerms;
        __syncwarp();
        if (lane < 5) reinterpret_cast<uint4 *>(&L)[lane] = reinterpret_cast<const uint4 *>(ix.lists + qt[0])[lane];
        __syncwarp();
        // decode the tile's keys: one fixed segment, or 1..255 consecutive
        // variable segments / one 256-slice of a large segment
        uint32_t kc = 0, first_elem;
        keys = s_keys[w];
        if (L.log2_block) {
            // tile ti: part (ti mod 2^s) of segment ti >> s; the whole segment is
            // decoded (d-gaps need its prefix) and the part's keys probed
            const uint32_t sp = tile_split_of(L.log2_block, b.tile_split);
            const uint32_t sg = L.seg_base + (ti >> sp);
            const uint32_t cnt = ix.seg_rec[sg].count;
            const uint32_t sub = (1u << L.log2_block) >> sp, e0 = (ti & ((1u << sp) - 1u)) * sub;
            first_elem = ((ti >> sp) << L.log2_block) + e0;
            warp_decode<KIND>(ix, L, sg, 0, cnt, keys, lane);
            kc = e0 < cnt ? min(sub, cnt - e0) : 0u;
            keys += e0;
        } else {
            const uint64_t tm = ix.tilemap[L.tile_base + ti];
            const uint32_t sg0 = L.seg_base + (uint32_t)(tm >> 32);
            const uint32_t e0 = (uint32_t)(tm >> 8) & kTileMaxE0, ns = (uint32_t)tm & 0xffu;
            first_elem = ix.seg_rec[sg0].start + e0;
            for (uint32_t g = 0; g < ns; ++g) {
                const uint32_t c = min(kTileKeys - kc, ix.seg_rec[sg0 + g].count - (g ? 0u : e0));
                warp_decode<KIND>(ix, L, sg0 + g, g ? 0u : e0, c, keys + kc, lane);
                kc += c;
            }
        }
        nkeys += kc;
        uint32_t alive = kc;
        for (uint32_t j = 1; j < k && alive; ++j) {
            __syncwarp();
            if (lane < 5) reinterpret_cast<uint4 *>(&L)[lane] = reinterpret_cast<const uint4 *>(ix.lists + qt[j])[lane];
            __syncwarp();
            // merge when the keys' range covers few segments: estimated from
            // the list's density first (no loads), then measured
            uint32_t span = 0, mseg0 = 0;
            if (b.merge_segs && alive >= kMergeMinKeys) {
                const uint32_t klo = keys[0], khi = keys[alive - 1];
                const double dens = (double)L.n / ((double)(L.last_doc - L.first_doc) + 1.0);
                if ((double)(khi - klo) * dens < 0.75 * kMergeCap) {
                    int sl = 0;
                    if (lane < 2) sl = locate_segment<ALGO>(ix, L, lane ? khi : klo);
                    const int s0 = max(__shfl_sync(0xffffffffu, sl, 0), 0), s1 = __shfl_sync(0xffffffffu, sl, 1);
                    if (s1 >= s0 && (uint32_t)(s1 - s0) < b.merge_segs) {
                        const uint32_t a0 = ix.seg_rec[L.seg_base + s0].start;
                        const SegRec r1 = ix.seg_rec[L.seg_base + s1];
                        if (r1.start + r1.count - a0 <= kMergeCap) {
                            span = r1.start + r1.count - a0;
                            mseg0 = (uint32_t)s0;
                            ++merges;
                            for (uint32_t sg = L.seg_base + s0; sg <= L.seg_base + (uint32_t)s1; ++sg) {
                                const SegRec r = ix.seg_rec[sg];
                                for (uint32_t e0 = 0; e0 < r.count; e0 += kTileKeys)
                                    warp_decode<KIND>(ix, L, sg, e0, min(kTileKeys, r.count - e0), mbuf + (r.start - a0) + e0,
                                                lane);
                            }
                        }
                    } else if (s1 < 0) {
                        alive = 0;  // every key precedes the list: nothing survives
                        continue;
                    }
                }
            }
            (void)mseg0;
            uint32_t nout = 0;
            // kProbeIlp keys per lane per round: keys base + 32k + lane
            for (uint32_t base = 0; base < alive; base += 32u * kProbeIlp) {
                uint32_t kv[kProbeIlp], act = 0;
#pragma unroll
                for (int k = 0; k < kProbeIlp; ++k) {
                    const uint32_t i = base + 32u * k + lane;
                    kv[k] = i < alive ? keys[i] : 0u;
                    act |= (uint32_t)(i < alive) << k;
                }
                uint32_t fm = 0;
                if (span) {
#pragma unroll
                    for (int k = 0; k < kProbeIlp; ++k) {
                        // first position with mbuf[pos] >= key, in shared memory
                        uint32_t lo = 0, hi = span;
                        while (lo < hi) {
                            const uint32_t mid = (lo + hi) >> 1;
                            if (mbuf[mid] < kv[k]) lo = mid + 1;
                            else hi = mid;
                        }
                        fm |= (uint32_t)((act >> k & 1u) && lo < span && mbuf[lo] == kv[k]) << k;
                    }
                } else {
                    fm = probe_keys<ALGO, KIND, kProbeIlp>(ix, L, kv, act, fallbacks);
                }
                probes += __popc(act);
                // every lane has read its keys before any survivor is written
                // back; groups are compacted in order, so survivors stay sorted
                __syncwarp();
#pragma unroll
                for (int k = 0; k < kProbeIlp; ++k) {
                    const bool f = fm >> k & 1u;
                    const uint32_t m = __ballot_sync(0xffffffffu, f);
                    if (f) keys[nout + __popc(m & ((1u << lane) - 1u))] = kv[k];
                    nout += __popc(m);
                }
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
        // nkeys and merges are warp-uniform: lane 0's count is the warp's
        if (lane == 0) {
            atomicAdd((unsigned long long *)&b.stats[0], (unsigned long long)probes);
            atomicAdd((unsigned long long *)&b.stats[1], (unsigned long long)fallbacks);
            atomicAdd((unsigned long long *)&b.stats[2], (unsigned long long)nkeys);
            atomicAdd((unsigned long long *)&b.stats[3], (unsigned long long)merges);
        }
    }
}

// ---------------------------------------------------------------------------
// Launchers.

template <int ALGO, int WARPS, int MINB, int KIND>
static void launch_probe_t(const DevIndexView &ix, const BatchView &b, int nsm, cudaStream_t st) {
    // persistent grid: as many CTAs as fit on the device at once, so every
    // resident warp pulls work items
    static int occ[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int per_sm = dev >= 0 && dev < 64 ? occ[dev] : 0;
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_probe<ALGO, WARPS, MINB, KIND>, WARPS * 32, 0);
        per_sm = per_sm > 0 ? per_sm : 1;
        if (dev >= 0 && dev < 64) occ[dev] = per_sm;
    }
    const uint32_t grid = (uint32_t)std::max(1, std::min(per_sm, (8 / WARPS) * MINB) * nsm);
    k_probe<ALGO, WARPS, MINB, KIND><<<grid, WARPS * 32, 0, st>>>(ix, b);
}

template <int ALGO, int WARPS, int MINB>
static void launch_probe_k(const DevIndexView &ix, const BatchView &b, int nsm, cudaStream_t st) {
    switch (codec_kind(ix.codec_mask)) {
        case kKindResid: launch_probe_t<ALGO, WARPS, MINB, kKindResid>(ix, b, nsm, st); break;
        case kKindDgap: launch_probe_t<ALGO, WARPS, MINB, kKindDgap>(ix, b, nsm, st); break;
        default: launch_probe_t<ALGO, WARPS, MINB, kKindAny>(ix, b, nsm, st); break;
    }
}

template <int WARPS, int MINB>
static void launch_probe_a(const DevIndexView &ix, const BatchView &b, int algo, int nsm, cudaStream_t st) {
    switch (algo) {
        case EXCL_ALGO_BSEARCH: launch_probe_k<EXCL_ALGO_BSEARCH, WARPS, MINB>(ix, b, nsm, st); break;
        case EXCL_ALGO_HASHSEG: launch_probe_k<EXCL_ALGO_HASHSEG, WARPS, MINB>(ix, b, nsm, st); break;
        case EXCL_ALGO_LEARNED: launch_probe_k<EXCL_ALGO_LEARNED, WARPS, MINB>(ix, b, nsm, st); break;
        default: launch_probe_k<EXCL_ALGO_AUTO, WARPS, MINB>(ix, b, nsm, st); break;
    }
}

template <int WARPS>
static void launch_probe_w(const DevIndexView &ix, const BatchView &b, int algo, int ctas_per_sm, int nsm,
                           cudaStream_t st) {
    // ctas_per_sm is counted in 8-warp CTAs
    if (ctas_per_sm <= 4) launch_probe_a<WARPS, 4>(ix, b, algo, nsm, st);
    else if (ctas_per_sm == 5) launch_probe_a<WARPS, 5>(ix, b, algo, nsm, st);
    else launch_probe_a<WARPS, 6>(ix, b, algo, nsm, st);
}

int launch_probe(const DevIndexView &ix, const BatchView &b, int algo, int warps, int ctas_per_sm, int nsm,
                 cudaStream_t st) {
    switch (warps) {
        case 4: launch_probe_w<4>(ix, b, algo, ctas_per_sm, nsm, st); break;
        default: launch_probe_w<8>(ix, b, algo, ctas_per_sm, nsm, st); break;
    }
    return (int)cudaGetLastError();
}

}  // namespace excl
