// sm_100a kernel of the batched AND-intersection path: one persistent launch
// per batch (k_batch) that packs the queries, probes, and scatters the
// results; this file holds its probe phase and the per-key search it runs
// against each longer list, batch_phases.cuh the pack and scatter phases.
// Whole-list decode is in decode.cu.
//
//   probe phase   each warp takes (query, tile) work items from an atomic
//                 queue, decodes the tile of the shortest list into smem,
//                 probes every longer list and compacts survivors with
//                 ballot/popc (replaces the search kernels, e.g.
//                 ParaPFD_Intersection_kernel.cu:145-458).
#include <cstdio>

#include "batch_phases.cuh"
#include "excl_device.cuh"
#include "kernels.h"

namespace excl {

// ---------------------------------------------------------------------------
// Probe of one key against one longer list.

__device__ __forceinline__ int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }
__device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

template <int ALGO, int KIND>
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
    // the segment: fixed blocks hold 2^log2_block postings, so a learned rank
    // window names its segments directly; a window inside one segment needs
    // no head search at all (a present key's rank lies in the window)
    const ProbeRec *pr = ix.seg_probe + L.seg_base;
    int s;
    if (learned) {
        lo = (uint32_t)(plo >> L.log2_block);
        hi = (uint32_t)(phi >> L.log2_block) + 1u;
        s = hi - lo == 1u ? (int)lo : last_head_le_rec(pr, lo, hi, key);
    } else if (ALGO == EXCL_ALGO_BSEARCH) {
        lo = 0;
        s = last_head_le(ix.seg_head + L.seg_base, 0, L.nseg, key);
    } else {
        const uint32_t b = (uint32_t)((uint64_t)key >> L.dir_shift);
        const uint32_t d0 = ldg(ix.dir + L.dir_base + b), d1 = ldg(ix.dir + L.dir_base + b + 1);
        lo = codec_is_hs(L.codec) ? d0 : (d0 ? d0 - 1u : 0u);
        hi = d1;
        s = last_head_le_rec(pr, lo, hi, key);
    }
    if (s < (int)lo) return false;
    // the segment's record: head, block offset, count, base/median, block
    // descriptor and segment regression
    const uint4 q0 = __ldg(reinterpret_cast<const uint4 *>(pr + s));
    const uint4 q1 = __ldg(reinterpret_cast<const uint4 *>(pr + s) + 1);
    SegRec rec;
    rec.off = q0.y;
    rec.aux = q0.z;
    rec.count = q0.w;
    const uint32_t *blk = ix.words + L.word_base + rec.off;
    const BlkHdr h = blk_hdr(q1.x);
    if (KIND == kKindAny && codec_is_newpfd(L.codec)) return dgap_find_newpfd(blk, h, rec.count, q0.x, rec.aux, key);
    if (KIND == kKindDgap || (KIND == kKindAny && codec_is_dgap(L.codec)))
        return dgap_find(blk, h, rec.count, q0.x, rec.aux, key);
    // list position of the segment: only learned windows and the LRC/LRCSeg
    // predictors use it, and those lists have fixed blocks
    rec.start = (uint32_t)s << L.log2_block;
    SegReg reg;
    reg.a = __uint_as_float(q1.y);
    reg.b = __uint_as_float(q1.z);
    reg.L = q1.w & 0xffffu;
    reg.R = q1.w >> 16;
    const ResidParams rp = resid_params(L, rec, reg);
    int64_t t0 = 0, t1 = (int64_t)rec.count - 1;
    if (learned) {
        t0 = imax64(t0, plo - rec.start);
        t1 = imin64(t1, phi - rec.start);
    } else if ((ALGO == EXCL_ALGO_SEGREG || ALGO == EXCL_ALGO_AUTO) &&
               (L.codec == EXCL_CODEC_SEGLRC || L.codec == EXCL_CODEC_HS_SEGLRC || L.codec == EXCL_CODEC_LRCSEG)) {
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
            rl = reg.L == kProbeUnbounded ? 0x7fffffffu : reg.L;
            rr = reg.R == kProbeUnbounded ? 0x7fffffffu : reg.R;
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
        const uint32_t d0 = ldg(ix.dir + L.dir_base + bk), d1 = ldg(ix.dir + L.dir_base + bk + 1);
        lo = codec_is_hs(L.codec) ? d0 : (d0 ? d0 - 1u : 0u);
        hi = d1;
    }
    return last_head_le(ix.seg_head + L.seg_base, lo, hi, key);
}

// ---------------------------------------------------------------------------
// The batch kernel: one persistent launch per batch (pack, probe, scatter;
// the pack and scatter phases are in batch_phases.cuh).
//
// Probe phase: for each longer list a tile chooses between two methods (the
// merge-path / probe choice): when the tile's surviving keys span few of the
// list's segments (at most b.merge_segs, whose docIDs fit kMergeCap), the warp
// decodes that span into shared memory once and every key is looked up there;
// otherwise each key is probed on its own (probe_key).

static_assert(kBatchWarps * 32 == kPackThreads && kBatchWarps * 32 == kSSThreads, "one CTA shape for every phase");

struct ProbeShared {
    uint32_t keys[kBatchWarps][kTileKeys];
    uint32_t merge[kBatchWarps][kMergeCap];
    ListDesc list[kBatchWarps];
};

// Spin limit of every cross-CTA wait: 2^22 polls, 32 ns to ~1 us of sleep
// each, so a wait that gives up has waited between 0.13 s and about 4 s.
constexpr uint32_t kSpin = 1u << 22;

// MINB: resident 8-warp CTAs per SM the register budget is cut for (4: 64
// registers; 5: 48; 6: 40), traded for more probes in flight; the launch
// shape is an autotuner choice. KIND: the codec family the instance handles
// (kKindAny for mixed indexes); a one-family instance needs fewer registers.
template <int ALGO, int MINB, int KIND>
__global__ void __launch_bounds__(kBatchWarps * 32, MINB) k_batch(const __grid_constant__ DevIndexView ix, const __grid_constant__ BatchView b, PackSync *sync,
                                                                  uint64_t *chunk_state, const ListDesc *lists,
                                                                  uint32_t nlists, const uint32_t *terms,
                                                                  const uint32_t *toff, uint32_t *offsets,
                                                                  uint32_t *docids, uint64_t cap, uint32_t spin) {
    __shared__ union {
        ProbeShared probe;
        PackShared pack;
        ScatterShared scatter;
    } sm;
    __shared__ uint32_t s_tag, s_ticket;
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    // every CTA reads the same epoch: it changes only when the last CTA of
    // this grid leaves, and that CTA has counted every other one out
    // the epoch read and the first pack ticket are in flight together
    if (threadIdx.x == 0) {
        const uint32_t e = *(volatile uint32_t *)&sync->epoch;
        s_ticket = atomicAdd(&sync->ticket, 1u);
        s_tag = next_tag(e);
    }
    __syncthreads();
    const uint32_t tag = s_tag;
    // failure-path self-test: a bounded wait on a flag that nothing sets gives
    // up and raises the expired-wait bit; the batch itself is unaffected
    if (b.check_polls && blockIdx.x == 0 && threadIdx.x == 0) wait_tag(b.check_flag, tag, b.err, b.check_polls);

    // ---- pack: chunks of qpc queries by ticket
    const uint32_t qpc = pack_chunk_queries(b.nq);
    const uint32_t npack = max(1u, (b.nq + qpc - 1) / qpc);
    for (bool first = true;; first = false) {
        if (!first && threadIdx.x == 0) s_ticket = atomicAdd(&sync->ticket, 1u);
        __syncthreads();
        const uint32_t bid = s_ticket;
        __syncthreads();
        if (bid >= npack) break;
        if (bid == 0 && threadIdx.x == 0 && b.stats) b.stats[4] = global_ns();
        pack_chunk(bid, npack, qpc, tag, lists, nlists, terms, toff, b.nq, b, sync, sm.pack, spin);
    }
    if (threadIdx.x == 0) {
        wait_packed(sync, npack, b.err, spin);
        if (b.stats) atomicMin((unsigned long long *)&b.stats[5], (unsigned long long)global_ns());
    }
    __syncthreads();

    // ---- probe. Work order: one record {tile, query, tile within the query,
    // shortest list} per tile in tile_order, heavy tiles from the front, the
    // others from the back. The records fill the first H and the last T - H
    // slots exactly, also after a tile overflow (reported as kErrCapacity),
    // where T is capped at max_tiles and the slots fill up.
    {
        uint32_t *keys = sm.probe.keys[w];  // the tile's keys (a sub-range of the decoded segment when tiles are cut)
        uint32_t *mbuf = sm.probe.merge[w];
        ListDesc &L = sm.probe.list[w];
        const uint32_t T = min(b.tile_prefix[b.nq], b.max_tiles);
        const uint32_t H = min(b.tile_prefix[b.nq + 1], T);
        uint32_t probes = 0, fallbacks = 0, nkeys = 0, merges = 0, done = 0;
        for (;;) {
            uint32_t wi = 0;
            if (lane == 0) wi = atomicAdd(b.tile_counter, 1u);
            wi = __shfl_sync(0xffffffffu, wi, 0);
            if (wi >= T) break;
            const uint4 wr = b.tile_order[wi < H ? wi : b.max_tiles - 1u - (wi - H)];
            const uint32_t t = wr.x, q = wr.y, ti = wr.z, list0 = wr.w;
            // the query's sorted terms (lane j holds term j), term count, key base
            // and the shortest list's descriptor: one round of independent loads
            const uint32_t tq = b.qterms[(size_t)q * kMaxTerms + lane];
            const uint32_t k = b.qnterms[q];
            const uint32_t kbase = b.key_base[q];
            __syncwarp();
            if (lane < 5) reinterpret_cast<uint4 *>(&L)[lane] = reinterpret_cast<const uint4 *>(ix.lists + list0)[lane];
            __syncwarp();
            // decode the tile's keys: one fixed segment, or 1..255 consecutive
            // variable segments / one 256-slice of a large segment
            uint32_t kc = 0, first_elem;
            keys = sm.probe.keys[w];
            if (L.log2_block) {
                // tile ti: part (ti mod 2^s) of segment ti >> s. Residual codecs
                // decode any element on its own, so only the part is decoded;
                // d-gap codecs decode the whole segment (the part needs its
                // prefix) and probe the part's keys
                const uint32_t sp = tile_split_of(L.log2_block, b.tile_split);
                const uint32_t sg = L.seg_base + (ti >> sp);
                // fixed blocks: every segment but the last holds 2^log2_block postings
                const uint32_t cnt = min(1u << L.log2_block, L.n - ((ti >> sp) << L.log2_block));
                const uint32_t sub = (1u << L.log2_block) >> sp, e0 = (ti & ((1u << sp) - 1u)) * sub;
                first_elem = ((ti >> sp) << L.log2_block) + e0;
                kc = e0 < cnt ? min(sub, cnt - e0) : 0u;
                const bool resid = KIND == kKindResid || (KIND == kKindAny && !codec_is_dgap(L.codec));
                if (sp && resid) {
                    if (kc) warp_decode<KIND>(ix, L, sg, e0, kc, keys, lane);
                } else {
                    warp_decode<KIND>(ix, L, sg, 0, cnt, keys, lane);
                    keys += e0;
                }
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
                const uint32_t lj = __shfl_sync(0xffffffffu, tq, j);
                __syncwarp();
                if (lane < 5) reinterpret_cast<uint4 *>(&L)[lane] = reinterpret_cast<const uint4 *>(ix.lists + lj)[lane];
                __syncwarp();
                // merge when the keys' range covers few segments: estimated from
                // the list's density first (no loads), then measured
                uint32_t span = 0;
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
                                ++merges;
                                for (uint32_t sg = L.seg_base + s0; sg <= L.seg_base + (uint32_t)s1; ++sg) {
                                    const SegRec r = ix.seg_rec[sg];
                                    for (uint32_t e0 = 0; e0 < r.count; e0 += kTileKeys)
                                        warp_decode<KIND>(ix, L, sg, e0, min(kTileKeys, r.count - e0),
                                                          mbuf + (r.start - a0) + e0, lane);
                                }
                            }
                        } else if (s1 < 0) {
                            alive = 0;  // every key precedes the list: nothing survives
                            continue;
                        }
                    }
                }
                uint32_t nout = 0;
                for (uint32_t base = 0; base < alive; base += 32) {
                    const uint32_t i = base + lane;
                    const bool valid = i < alive;
                    const uint32_t key = valid ? keys[i] : 0u;
                    bool f;
                    if (span) {
                        // first position with mbuf[pos] >= key, in shared memory
                        uint32_t lo = 0, hi = span;
                        while (lo < hi) {
                            const uint32_t mid = (lo + hi) >> 1;
                            if (mbuf[mid] < key) lo = mid + 1;
                            else hi = mid;
                        }
                        f = valid && lo < span && mbuf[lo] == key;
                    } else {
                        f = valid && probe_key<ALGO, KIND>(ix, L, key, fallbacks);
                    }
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
            const uint64_t slot = (uint64_t)kbase + first_elem;
            if (slot + kc > b.max_keys) {
                if (lane == 0) atomicOr(b.err, kErrCapacity);
                alive = 0;
            }
            uint32_t *dst = b.scratch + slot;
            for (uint32_t i = lane; i < alive; i += 32) dst[i] = keys[i];
            if (lane == 0) {
                b.tile_count[t] = alive;
                b.tile_slot[t] = (uint32_t)slot;
                b.tile_q[t] = ti == 0 ? q + 1u : 0u;  // first-tile mark for the scatter phase's offsets
            }
            ++done;
            __syncwarp();
        }
        // this warp's tiles are written: count them in (the scatter phase
        // starts when the count reaches the batch's tiles)
        __threadfence();
        __syncwarp();
        if (lane == 0) {
            if (done) red_release_add(b.probe_done, done);
            if (b.stats) atomicMax((unsigned long long *)&b.stats[6], (unsigned long long)global_ns());
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
    __syncthreads();  // the shared union passes to the scatter phase

    // ---- scatter
    scatter_phase(b, sync, chunk_state, offsets, docids, cap, tag, sm.scatter, spin);

    // the last CTA out resets the counters, hands the batch's error bits to
    // the host and passes the epoch on; every thread's writes are fenced
    // before its CTA counts itself out
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0 && atomicAdd(&sync->sdone, 1u) == gridDim.x - 1) {
        __threadfence();
        sync->ticket = 0u;
        sync->sticket = 0u;
        sync->sdone = 0u;
        sync->packed = 0u;
        if (b.stats) b.stats[7] = global_ns();
        hand_over_flags(b);
        sync->epoch = tag;
        __threadfence();
    }
}

// ---------------------------------------------------------------------------
// Launchers.

template <int ALGO, int MINB, int KIND>
static cudaError_t launch_batch_t(const BatchLaunch &L, cudaStream_t st) {
    // persistent grid: as many CTAs as fit on the device at once, so every
    // resident warp pulls work items
    static int occ[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int per_sm = dev >= 0 && dev < 64 ? occ[dev] : 0;
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<ALGO, MINB, KIND>, kBatchWarps * 32, 0);
        per_sm = per_sm > 0 ? per_sm : 1;
        if (dev >= 0 && dev < 64) occ[dev] = per_sm;
    }
    // a small batch (its tile count known on the host) takes one warp per
    // tile, so the batches of other streams keep the rest of the device
    uint32_t grid = (uint32_t)std::max(1, std::min(per_sm, MINB) * L.nsm);
    if (L.max_ctas) grid = std::min(grid, L.max_ctas);
    k_batch<ALGO, MINB, KIND><<<grid, kBatchWarps * 32, 0, st>>>(L.ixv, L.b, L.sync, L.chunk_state, L.lists, L.nlists,
                                                                  L.terms, L.toff, L.offsets, L.docids, L.cap,
                                                                  L.spin ? L.spin : kSpin);
    return cudaGetLastError();
}

template <int ALGO, int MINB>
static cudaError_t launch_batch_k(const BatchLaunch &L, cudaStream_t st) {
    switch (codec_kind(L.ixv.codec_mask)) {
        case kKindResid: return launch_batch_t<ALGO, MINB, kKindResid>(L, st);
        case kKindDgap: return launch_batch_t<ALGO, MINB, kKindDgap>(L, st);
        default: return launch_batch_t<ALGO, MINB, kKindAny>(L, st);
    }
}

template <int MINB>
static cudaError_t launch_batch_a(const BatchLaunch &L, cudaStream_t st) {
    switch (L.algo) {
        case EXCL_ALGO_BSEARCH: return launch_batch_k<EXCL_ALGO_BSEARCH, MINB>(L, st);
        case EXCL_ALGO_HASHSEG: return launch_batch_k<EXCL_ALGO_HASHSEG, MINB>(L, st);
        case EXCL_ALGO_LEARNED: return launch_batch_k<EXCL_ALGO_LEARNED, MINB>(L, st);
        case EXCL_ALGO_SEGREG: return launch_batch_k<EXCL_ALGO_SEGREG, MINB>(L, st);
        default: return launch_batch_k<EXCL_ALGO_AUTO, MINB>(L, st);
    }
}

int launch_batch(const BatchLaunch &L, cudaStream_t st) {
    if (L.b.nq > kPackMaxQueries) return (int)cudaErrorInvalidValue;
    if (L.ev) cudaEventRecord(L.ev[0], st);
    // ctas_per_sm is counted in 8-warp CTAs
    cudaError_t e;
    if (L.ctas_per_sm <= 4) e = launch_batch_a<4>(L, st);
    else if (L.ctas_per_sm == 5) e = launch_batch_a<5>(L, st);
    else e = launch_batch_a<6>(L, st);
    if (L.ev) {
        cudaEventRecord(L.ev[1], st);
        cudaEventRecord(L.ev[2], st);
        cudaEventRecord(L.ev[3], st);
    }
    return (int)e;
}

}  // namespace excl
