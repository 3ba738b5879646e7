// K1/K2 whole-list decode with TMA bulk staging.
//
// Each CTA owns a contiguous range of segments. Consecutive ParaPFD blocks are
// contiguous in the index's word array, so a run of up to 32 segments is one
// contiguous byte range: warp 0 plans the next run (32 segments' metadata
// loaded 32-wide, a ballot finds how many fit a 24 KB stage), and one
// cp.async.bulk copies the run into shared memory, completing on an mbarrier,
// while all warps decode the previous run from the other stage. Decoding works
// from shared memory only: bit-window extraction of each lane's values,
// exception patching, d-gap scan (ParaPFD_Decompression_kernel.cu:205-263)
// or regression reconstruction (SegLRC_Decompression_kernel.cu:249-252), then
// stores. A segment of c values takes G lanes (the smallest power of two with
// c <= 8G), so one warp decodes 32/G short segments at once: a segment's
// fixed cost (header, scan, synchronisation) is shared instead of paid by a
// whole warp for a handful of postings. Hash buckets of more than 256 postings are not
// staged; their 256-slices are decoded from global memory.
//
// No multicast is used: each CTA copies only into its own shared memory.
#include <cuda_runtime.h>

#include "excl_device.cuh"
#include "kernels.h"

namespace excl {

#ifndef EXCL_DEC_WARPS
#define EXCL_DEC_WARPS 4
#endif
#ifndef EXCL_DEC_STAGES
#define EXCL_DEC_STAGES 2
#endif
#ifndef EXCL_DEC_STAGE_WORDS
#define EXCL_DEC_STAGE_WORDS 2048
#endif
#ifndef EXCL_DEC_CTAS_PER_SM
#define EXCL_DEC_CTAS_PER_SM 8
#endif
constexpr int kDecWarps = EXCL_DEC_WARPS;
constexpr uint32_t kStages = EXCL_DEC_STAGES;         // ring of staged runs: copies in flight while one is decoded
constexpr uint32_t kStageCap = EXCL_DEC_STAGE_WORDS;  // words per stage (a run of 32 segments needs ~3-13 KB; longer runs are cut)
constexpr int kDecCtasPerSm = EXCL_DEC_CTAS_PER_SM;
static_assert(kStageCap >= 1024, "a stage holds at least one block of 256 values at 32 bits plus exceptions");
constexpr uint32_t kDecChunk = 64;  // segments per work ticket
constexpr uint32_t kRunSegs = 32;
constexpr uint32_t kWaitLimit = 1u << 22;  // try_wait polls before giving up (a stage normally lands in microseconds)

struct alignas(16) RunMeta {
    uint64_t ob;       // output position of the segment's first docID
    uint32_t woff;     // descriptor word within the stage
    uint32_t count, start, aux, head, list;
    float a, b;
    uint32_t codec, r0, r1;  // the list's codec and list-level regression words
    uint32_t bw;             // the block's words
    uint32_t pad[2];
};

struct DecodeSmem {
    uint32_t stage[kStages][kStageCap + 8];
    RunMeta meta[kStages][kRunSegs];
    uint32_t vals[kDecWarps][kTileKeys + kTileKeys / 32];
    unsigned long long mbar[kStages];
    uint32_t run_n[kStages];       // segments in the run
    uint32_t run_big[kStages];     // 1: a single large bucket, not staged
    uint32_t run_first[kStages];   // global index of the run's first segment
    uint32_t have[kStages];        // 1: stage holds a planned run
    // units of the run: unit u decodes useg[u][0 .. ucnt[u]) (indexes into meta),
    // all of width class ucls[u] (d-gap or residual, log2 of the lanes per segment)
    uint8_t useg[kStages][kRunSegs][kRunSegs];
    uint8_t ucls[kStages][kRunSegs];
    uint8_t ucnt[kStages][kRunSegs];
    uint32_t nunits[kStages];
    uint32_t unext[kStages];  // next unit to claim
    uint32_t next_seg;       // first segment not yet planned in the current chunk
    uint32_t chunk_end;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Warp 0: plan the run starting at segment s0 (< se) into stage b and start its copy.
__device__ void plan_run(const DevIndexView &ix, DecodeSmem &sm, uint32_t b, uint32_t s0, uint32_t se,
                         uint64_t out_base0, uint32_t lane) {
    const uint32_t s = s0 + lane;
    const bool valid = s < se;
    uint32_t l = 0, count = 0, start = 0, aux = 0, head = 0, codec = 0, r0 = 0, r1 = 0;
    uint64_t gword = 0, bw = 0, ob = 0;
    float a = 1.0f, bb = 0.0f;
    if (valid) {
        // independent loads, one round trip: the segment's 64-byte probe
        // record (which carries its list's codec, regression words and output
        // position), its block's word range and its list id
        const uint4 *pr = reinterpret_cast<const uint4 *>(ix.seg_probe + s);
        const uint4 p0 = __ldg(pr), p1 = __ldg(pr + 1), p2 = __ldg(pr + 2), p3 = __ldg(pr + 3);
        gword = ix.seg_gword[s];
        bw = ix.seg_gword[s + 1] - gword;
        l = ix.seg_list[s];
        head = p0.x;
        aux = p0.z;
        count = p0.w;
        a = __uint_as_float(p1.y);
        bb = __uint_as_float(p1.z);
        start = p2.x;
        codec = p2.y;
        ob = ((uint64_t)p2.w << 32 | p2.z) - out_base0;
        r0 = p3.x;
        r1 = p3.y;
    }
    const bool big = valid && count > kTileKeys;
    const uint64_t base = __shfl_sync(0xffffffffu, gword, 0) & ~3ull;  // 16-byte aligned start
    // words to copy if this lane's segment closes the run (+4 so the bit window may read one word past a block)
    const uint64_t need = ((gword + bw + 4 + 3) & ~3ull) - base;
    const bool fits = valid && !big && need <= kStageCap;
    const uint32_t bad = __ballot_sync(0xffffffffu, !fits);
    const bool first_big = __shfl_sync(0xffffffffu, big, 0);
    uint32_t n = first_big ? 1u : (bad ? (uint32_t)(__ffs(bad) - 1) : 32u);
    if (n == 0) n = 1;  // unreachable for valid blocks (<= 561 words); keeps progress
    if (lane < n) {
        RunMeta &m = sm.meta[b][lane];
        m.ob = ob;
        m.woff = (uint32_t)(gword - base);
        m.count = count;
        m.start = start;
        m.aux = aux;
        m.head = head;
        m.list = l;
        m.a = a;
        m.b = bb;
        m.codec = codec;
        m.r0 = r0;
        m.r1 = r1;
        m.bw = (uint32_t)bw;
    }
    // width classes: a segment of c values takes G = 2^lg lanes, the smallest
    // power of two with c <= 8G, and 32/G segments of one class (same kind,
    // same G) share a warp; a lane's rank among its class's segments gives its unit
    const uint32_t need_lanes = (count + 7u) >> 3;
    const uint32_t lg = need_lanes <= 1u ? 0u : 32u - __clz(need_lanes - 1u);
    const uint32_t cls = lane < n ? (codec_is_dgap(codec) ? 0u : 6u) + lg : 0xffu;
    uint32_t nunits = 0;
#pragma unroll
    for (uint32_t c = 0; c < 12; ++c) {
        const uint32_t mk = __ballot_sync(0xffffffffu, cls == c);
        const uint32_t per = 32u >> (c % 6u), tot = __popc(mk);
        if (cls == c) {
            const uint32_t rank = __popc(mk & ((1u << lane) - 1u));
            const uint32_t u = nunits + rank / per, slot = rank % per;
            sm.useg[b][u][slot] = (uint8_t)lane;
            if (slot == 0) {
                sm.ucls[b][u] = (uint8_t)c;
                sm.ucnt[b][u] = (uint8_t)min(per, tot - rank);
            }
        }
        nunits += (tot + per - 1u) / per;
    }
    const uint64_t need_last = __shfl_sync(0xffffffffu, need, n - 1);
    if (lane == 0) {
        sm.nunits[b] = nunits;
        sm.unext[b] = 0;
        sm.run_n[b] = n;
        sm.run_big[b] = first_big ? 1u : 0u;
        sm.run_first[b] = s0;
        sm.next_seg = s0 + n;
        if (!first_big) {
            const uint32_t bytes = (uint32_t)need_last * 4u;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&sm.mbar[b], bytes);
            bulk_g2s(sm.stage[b], ix.words + base, bytes, &sm.mbar[b]);
        }
    }
    __syncwarp();
}

// Group widths are template arguments (unrolled scans and strides) or, for
// kLgRuntime, a run-time value (one body for every width: less code).
constexpr uint32_t kLgRuntime = 8;
#ifndef EXCL_DEC_DGAP_FIXED
#define EXCL_DEC_DGAP_FIXED 0
#endif
#ifndef EXCL_DEC_RESID_FIXED
#define EXCL_DEC_RESID_FIXED 1
#endif

// A warp's value buffer holds warp-relative element i at word i + i/32, so
// lanes storing runs of 2, 4 or 8 consecutive values hit distinct banks.
__device__ __forceinline__ uint32_t sw(uint32_t i) { return i + (i >> 5); }

// Exceptions of a staged ParaPFD block (ParaPFor.cpp:112-123): the G = 2^lg
// lanes of a group patch the high bits of the listed positions into the
// group's values, element i at vals[sw(base + i)]. Positions are distinct, so
// the lanes never write the same word.
__device__ __forceinline__ void group_patch(const uint32_t *lows, BlkHdr h, uint32_t count, uint32_t *vals,
                                            uint32_t base, uint32_t lg, uint32_t sub) {
    const uint32_t *pb = lows + words_for(count, h.lb);
    const uint32_t *hp = pb + words_for(h.en, h.eb);
    for (uint32_t x = sub; x < h.en; x += 1u << lg) {
        const uint32_t pbit = x * h.eb, hbit = x * h.hb;
        const uint32_t p = __funnelshift_r(pb[pbit >> 5], pb[(pbit >> 5) + 1], pbit & 31u) & ((1u << h.eb) - 1u);
        const uint32_t hv = __funnelshift_r(hp[hbit >> 5], hp[(hbit >> 5) + 1], hbit & 31u) & ((1u << h.hb) - 1u);
        if (p < count) vals[sw(base + p)] |= hv << h.lb;
    }
}

// d-gap codecs, one segment per group of G = 2^lg lanes (count <= 8G):
// lane `sub` owns a run of ceil(count/G) consecutive values; the segment head
// replaces value 0, then a G-wide scan turns gaps into docIDs
// (ParaPFD_Decompression_kernel.cu:205-263) and the group stores its values
// G-wide from the warp's buffer. Inactive groups (act false) run the same
// warp-wide steps on count 0. Every lane of the warp passes the same lg.
template <uint32_t LGT>
__device__ __forceinline__ void group_dgap(const uint32_t *blk, const RunMeta &m, bool act, uint32_t lg_rt,
                                           uint32_t sub, uint32_t *vals, uint32_t base, uint32_t *__restrict__ out) {
    const uint32_t lg = LGT == kLgRuntime ? lg_rt : LGT;
    const uint32_t G = 1u << lg;
    const BlkHdr h = blk_hdr(blk[0]);
    const uint32_t *lows = blk + 1;
    const uint32_t count = act ? m.count : 0u;
    const uint32_t vpl = (count + G - 1u) >> lg;
    const uint32_t el = sub * vpl;
    const uint32_t mask = (1u << h.lb) - 1u;
    uint32_t v[8];
    {
        // a 64-bit window slides over the lane's words (as group_dgap_full),
        // moving on only while the lane has another value to extract
        const uint32_t nv = el < count ? min(vpl, count - el) : 0u;
        const uint32_t bit0 = el * h.lb;
        uint32_t wi = bit0 >> 5, sh = bit0 & 31u;
        uint32_t lo = nv ? lows[wi] : 0u, hi = nv ? lows[wi + 1] : 0u;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            v[q] = q < (int)nv ? (__funnelshift_r(lo, hi, sh) & mask) : 0u;
            sh += h.lb;
            if (q + 1 < (int)nv && sh >= 32u) {
                sh -= 32u;
                lo = hi;
                ++wi;
                hi = lows[wi + 1];
            }
        }
    }
    const bool exc = count && h.en;
    if (__any_sync(0xffffffffu, exc)) {
        if (exc) {
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (q < (int)vpl && el + q < count) vals[sw(base + el + q)] = v[q];
        }
        __syncwarp();
        // NewPFD blocks: their groups decode the Simple-16 exception stream
        // together (every lane of the warp takes part in the shuffles)
        const bool npfd = exc && codec_is_newpfd(m.codec);
        if (__any_sync(0xffffffffu, npfd))
            newpfd_patch_group(lows + words_for(count, h.lb), npfd ? m.bw - 1u - words_for(count, h.lb) : 0u,
                               npfd ? h.en : 0u, h.lb, 0u, count, lg, sub,
                               [vals, base](uint32_t i) -> uint32_t & { return vals[sw(base + i)]; });
        if (exc && !npfd) group_patch(lows, h, count, vals, base, lg, sub);
        __syncwarp();
        if (exc) {
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (q < (int)vpl && el + q < count) v[q] = vals[sw(base + el + q)];
        }
        __syncwarp();
    }
    if (sub == 0) v[0] = count ? m.head : 0u;
    uint32_t run = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        run += v[q];
        v[q] = run;
    }
    uint32_t incl = run;
#pragma unroll
    for (uint32_t o = 1; o < G; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o, G);
        if (sub >= o) incl += t;
    }
    const uint32_t ex = incl - run;
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (q < (int)vpl && el + q < count) vals[sw(base + el + q)] = v[q] + ex;
    __syncwarp();
    uint32_t *o = out + m.ob;
    for (uint32_t i = sub; i < count; i += G) o[i] = vals[sw(base + i)];
    __syncwarp();
}

// d-gap codecs, full blocks of 8G values with G = 16 or 32 (ParaPFD blocks of
// 128 or 256): the same steps as group_dgap with every bound known, so no
// value needs a bounds test, the G-wide scan is unrolled, and each lane's
// eight consecutive docIDs leave its registers as two 16-byte stores when the
// group's output is 16-byte aligned. Every group of the warp holds such a
// block.
template <uint32_t LG>
__device__ __forceinline__ void group_dgap_full(const uint32_t *blk, const RunMeta &m, uint32_t sub, uint32_t *vals,
                                                uint32_t base, uint32_t *__restrict__ out) {
    constexpr uint32_t G = 1u << LG, count = 8u * G;
    const BlkHdr h = blk_hdr(blk[0]);
    const uint32_t *lows = blk + 1;
    const uint32_t mask = (1u << h.lb) - 1u;
    const uint32_t el = sub * 8u;
    uint32_t v[8];
    // a 64-bit window slides over the lane's words: each word is read from
    // shared memory once (two words, then one more whenever the bit position
    // crosses a word) instead of twice per value
    const uint32_t bit0 = el * h.lb;
    uint32_t wi = bit0 >> 5, sh = bit0 & 31u;
    uint32_t lo = lows[wi], hi = lows[wi + 1];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        v[q] = __funnelshift_r(lo, hi, sh) & mask;
        sh += h.lb;
        if (q < 7 && sh >= 32u) {
            sh -= 32u;
            lo = hi;
            ++wi;
            hi = lows[wi + 1];
        }
    }
    const bool exc = h.en != 0;
    if (__any_sync(0xffffffffu, exc)) {
        if (exc) {
#pragma unroll
            for (int q = 0; q < 8; ++q) vals[sw(base + el + q)] = v[q];
        }
        __syncwarp();
        const bool npfd = exc && codec_is_newpfd(m.codec);
        if (__any_sync(0xffffffffu, npfd))
            newpfd_patch_group(lows + words_for(count, h.lb), npfd ? m.bw - 1u - words_for(count, h.lb) : 0u,
                               npfd ? h.en : 0u, h.lb, 0u, count, LG, sub,
                               [vals, base](uint32_t i) -> uint32_t & { return vals[sw(base + i)]; });
        if (exc && !npfd) group_patch(lows, h, count, vals, base, LG, sub);
        __syncwarp();
        if (exc) {
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = vals[sw(base + el + q)];
        }
        __syncwarp();
    }
    if (sub == 0) v[0] = m.head;
    uint32_t run = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        run += v[q];
        v[q] = run;
    }
    uint32_t incl = run;
#pragma unroll
    for (uint32_t o = 1; o < G; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o, G);
        if (sub >= o) incl += t;
    }
    const uint32_t ex = incl - run;
    // a group whose output starts on a 16-byte boundary stores its lanes'
    // eight docIDs as two 16-byte vectors; another (a hash bucket's block
    // starts anywhere) goes through the warp's buffer and stores G-wide
    uint32_t *ob = out + m.ob;
    const bool al = (reinterpret_cast<uintptr_t>(ob) & 15u) == 0;
    if (__all_sync(0xffffffffu, al)) {
        uint4 *o = reinterpret_cast<uint4 *>(ob + el);
        o[0] = make_uint4(v[0] + ex, v[1] + ex, v[2] + ex, v[3] + ex);
        o[1] = make_uint4(v[4] + ex, v[5] + ex, v[6] + ex, v[7] + ex);
        return;
    }
    if (!al) {
#pragma unroll
        for (int q = 0; q < 8; ++q) vals[sw(base + el + q)] = v[q] + ex;
    }
    __syncwarp();
    if (al) {
        uint4 *o = reinterpret_cast<uint4 *>(ob + el);
        o[0] = make_uint4(v[0] + ex, v[1] + ex, v[2] + ex, v[3] + ex);
        o[1] = make_uint4(v[4] + ex, v[5] + ex, v[6] + ex, v[7] + ex);
    } else {
#pragma unroll
        for (uint32_t j = 0; j < 8; ++j) ob[sub + G * j] = vals[sw(base + sub + G * j)];
    }
    __syncwarp();
}

// Residual codecs (LRC, LRCSeg, SegLRC, HS_SegLRC), one segment per group of
// G lanes: no scan; lane `sub` owns values sub, sub+G, ... so the group reads
// neighbouring words and every value goes from its register straight into a
// G-wide store. Reconstruction as the reference:
// LRC_Decompression_kernel.cu:254, SegLRC_Decompression_kernel.cu:252.
template <uint32_t LGT>
__device__ __forceinline__ void group_resid(const uint32_t *blk, const RunMeta &m, bool act, uint32_t lg_rt,
                                            uint32_t sub, uint32_t *vals, uint32_t base,
                                            uint32_t *__restrict__ out) {
    const uint32_t lg = LGT == kLgRuntime ? lg_rt : LGT;
    const uint32_t G = 1u << lg;
    const BlkHdr h = blk_hdr(blk[0]);
    const uint32_t *lows = blk + 1;
    const uint32_t count = act ? m.count : 0u;
    const uint32_t mask = (1u << h.lb) - 1u;
    uint32_t v[8];
    if (LGT == 5) {
        // G = 32: value t = sub + 32q starts at bit sub*lb + 32*q*lb, so its
        // word is q*lb words past the lane's first one and its shift is the
        // lane's own; a full block needs no bounds test
        const uint32_t b0 = sub * h.lb, sh = b0 & 31u;
        const uint32_t *p = lows + (b0 >> 5);
        if (count == 8u * 32u) {
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = __funnelshift_r(p[q * h.lb], p[q * h.lb + 1], sh) & mask;
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q)
                v[q] = sub + 32u * q < count ? (__funnelshift_r(p[q * h.lb], p[q * h.lb + 1], sh) & mask) : 0u;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t t = sub + G * q;
            const uint32_t bit = t * h.lb;
            const uint32_t wi = bit >> 5;
            v[q] = t < count ? (__funnelshift_r(lows[wi], lows[wi + 1], bit & 31u) & mask) : 0u;
        }
    }
    const bool exc = count && h.en;
    if (__any_sync(0xffffffffu, exc)) {
        if (exc) {
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (sub + G * q < count) vals[sw(base + sub + G * q)] = v[q];
        }
        __syncwarp();
        if (exc) group_patch(lows, h, count, vals, base, lg, sub);
        __syncwarp();
        if (exc) {
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (sub + G * q < count) v[q] = vals[sw(base + sub + G * q)];
        }
        __syncwarp();
    }
    uint32_t *o = out + m.ob;
    if (m.codec == EXCL_CODEC_LRC) {
        const float slope = __uint_as_float(m.r0);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t t = sub + G * q;
            if (t < count) o[t] = v[q] + pred_lrc(m.start + t, slope, (int32_t)m.r1);
        }
    } else if (m.codec == EXCL_CODEC_LRCSEG) {
        // list-level index: the float conversion of start + t as the reference's
        const float a = __uint_as_float(m.r0), b = __uint_as_float(m.r1);
        const uint32_t aux = m.aux, i0 = m.start;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t t = sub + G * q;
            if (t < count) o[t] = v[q] + pred_fma(i0 + t, a, b) + aux;
        }
    } else {
        // segment-local index t < 256: float(sub) + G*q is exact, so one
        // conversion per lane replaces one per value
        const float a = m.a, b = m.b;
        const uint32_t aux = m.aux;
        const float tf = __uint2float_rn(sub);
        if (LGT == 5 && count == 8u * 32u) {
#pragma unroll
            for (int q = 0; q < 8; ++q)
                o[sub + 32u * q] = v[q] + (uint32_t)__float2int_rz(__fmaf_rn(__fadd_rn(tf, 32.0f * q), a, b)) + aux;
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t t = sub + G * q;
                const float tq = __fadd_rn(tf, (float)(G * q));
                if (t < count) o[t] = v[q] + (uint32_t)__float2int_rz(__fmaf_rn(tq, a, b)) + aux;
            }
        }
    }
}

// Warp 0: the next chunk of segments from the work counter (false: none left).
__device__ __forceinline__ bool grab_chunk(uint32_t *tk, uint32_t nchunks, uint32_t seg0, uint32_t seg_end,
                                           uint32_t lane, uint32_t &s0, uint32_t &se) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(tk, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunks) return false;
    s0 = seg0 + c * kDecChunk;
    se = min(s0 + kDecChunk, seg_end);
    return true;
}

// Persistent: CTAs take chunks of kDecChunk segments from a counter (so long
// and short lists balance), warp 0 plans and copies run k+1 while all warps
// decode run k. tk[0] is the chunk counter, tk[1] counts finished CTAs; the
// last CTA out resets both.
__global__ void __launch_bounds__(kDecWarps * 32, kDecCtasPerSm) k_decode_tma(DevIndexView ix, uint32_t l0, uint32_t l1,
                                                                              uint64_t out_base0,
                                                                              uint32_t *__restrict__ out,
                                                                              uint32_t seg0, uint32_t nsegs,
                                                                              uint32_t *tk, uint32_t *err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    DecodeSmem &sm = *reinterpret_cast<DecodeSmem *>(smem_raw);
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t seg_end = seg0 + nsegs;
    const uint32_t nchunks = (nsegs + kDecChunk - 1) / kDecChunk;
    if (threadIdx.x == 0) {
        for (uint32_t k = 0; k < kStages; ++k) mbar_init(&sm.mbar[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // warp 0 plans runs in order into the ring; plan_next fills stage k
    uint32_t p_next = 0, p_end = 0;  // warp 0's position in its current chunk
    auto plan_next = [&](uint32_t k) {
        uint32_t s0 = p_next, se = p_end;
        const bool ok = s0 < se || grab_chunk(tk, nchunks, seg0, seg_end, lane, s0, se);
        if (ok) {
            plan_run(ix, sm, k, s0, se, out_base0, lane);
            p_next = sm.next_seg;
            p_end = se;
        }
        if (lane == 0) sm.have[k] = ok;
        __syncwarp();
    };
    if (w == 0)
        for (uint32_t k = 0; k + 1 < kStages; ++k) plan_next(k);
    __syncthreads();
    uint32_t phase[kStages] = {};
    bool failed = false;
    const bool any = sm.have[0] != 0;  // this CTA got a chunk
    for (uint32_t it = 0; any; ++it) {
        const uint32_t b = it % kStages;
        const uint32_t big = sm.run_big[b], first = sm.run_first[b];
        __syncthreads();  // everyone has read the run header before warp 0 refills the ring
        if (w == 0) plan_next((it + kStages - 1) % kStages);  // the stage decoded in the previous iteration
        if (big) {
            // one large hash bucket: 256-slices from global memory, spread over the warps
            const RunMeta &m = sm.meta[b][0];
            const ListDesc L = ix.lists[m.list];
            for (uint32_t e0 = w * kTileKeys; e0 < m.count; e0 += kDecWarps * kTileKeys) {
                const uint32_t kc = min(kTileKeys, m.count - e0);
                warp_decode(ix, L, first, e0, kc, sm.vals[w], lane);
                for (uint32_t i = lane; i < kc; i += 32) out[m.ob + e0 + i] = sm.vals[w][i];
                __syncwarp();
            }
        } else {
            uint32_t spins = 0;
            while (!mbar_try_wait(&sm.mbar[b], phase[b])) {
                if (++spins > kWaitLimit) {
                    failed = true;
                    break;
                }
            }
            phase[b] ^= 1u;
            // units are claimed from a shared counter, so warp 0, which planned
            // the next run first, decodes fewer of them when planning ran long
            if (!failed)
                for (;;) {
                    uint32_t u = 0;
                    if (lane == 0) u = atomicAdd(&sm.unext[b], 1u);
                    u = __shfl_sync(0xffffffffu, u, 0);
                    if (u >= sm.nunits[b]) break;
                    // unit u: group grp of G = 2^lg lanes takes the unit's grp-th segment
                    const uint32_t c = sm.ucls[b][u], lg = c % 6u;
                    const uint32_t grp = lane >> lg, sub = lane & ((1u << lg) - 1u);
                    const bool act = grp < sm.ucnt[b][u];
                    const RunMeta &m = sm.meta[b][sm.useg[b][u][act ? grp : 0u]];
                    const uint32_t base = grp * (8u << lg);
                    const uint32_t *blk = sm.stage[b] + m.woff;
                    uint32_t *vals = sm.vals[w];
#define EXCL_DEC_CALL(F, L) F<L>(blk, m, act, lg, sub, vals, base, out)
#define EXCL_DEC_SWITCH(F)                                  \
    switch (lg) {                                           \
        case 0: EXCL_DEC_CALL(F, 0); break;                 \
        case 1: EXCL_DEC_CALL(F, 1); break;                 \
        case 2: EXCL_DEC_CALL(F, 2); break;                 \
        case 3: EXCL_DEC_CALL(F, 3); break;                 \
        case 4: EXCL_DEC_CALL(F, 4); break;                 \
        default: EXCL_DEC_CALL(F, 5); break;                \
    }
                    if (c < 6u) {
                        // full blocks of 128 or 256 values in every group
                        const bool full = act && (lg == 4u || lg == 5u) && m.count == (8u << lg);
                        if (__all_sync(0xffffffffu, full)) {
                            if (lg == 4u) group_dgap_full<4>(blk, m, sub, vals, base, out);
                            else group_dgap_full<5>(blk, m, sub, vals, base, out);
                        } else if (EXCL_DEC_DGAP_FIXED) {
                            EXCL_DEC_SWITCH(group_dgap)
                        } else {
                            EXCL_DEC_CALL(group_dgap, kLgRuntime);
                        }
                    } else {
                        if (EXCL_DEC_RESID_FIXED) { EXCL_DEC_SWITCH(group_resid) }
                        else EXCL_DEC_CALL(group_resid, kLgRuntime);
                    }
#undef EXCL_DEC_SWITCH
#undef EXCL_DEC_CALL
                }
        }
        __syncthreads();  // stage b and its metadata are free again; the newly planned header is visible
        if (__syncthreads_or(failed)) {
            // a copy never landed: flag it, give the copies still in flight a
            // bounded chance to land, and stop
            if (threadIdx.x == 0) {
                atomicOr(err, kErrScanSpin);
                for (uint32_t d = 1; d < kStages; ++d) {
                    const uint32_t o = (it + d) % kStages;
                    if (sm.have[o] && !sm.run_big[o])
                        for (uint32_t k = 0; k < kWaitLimit && !mbar_try_wait(&sm.mbar[o], phase[o]); ++k) {
                        }
                }
            }
            break;
        }
        if (!sm.have[(it + 1) % kStages]) break;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(tk + 1, 1u) == gridDim.x - 1) {
            tk[0] = 0u;
            tk[1] = 0u;
            __threadfence();
        }
    }
}

int launch_decode(const DevIndexView &ix, uint32_t l0, uint32_t l1, uint64_t out_base0, uint32_t *out, uint32_t seg0,
                  uint32_t nsegs, int nsm, uint32_t *tk, uint32_t *err, cudaStream_t st) {
    if (nsegs == 0) return 0;
    static bool attr_set[64] = {};
    const size_t smem = sizeof(DecodeSmem);
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k_decode_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
    const uint64_t nchunks = (nsegs + kDecChunk - 1) / kDecChunk;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(nchunks, (uint64_t)nsm * kDecCtasPerSm));
    k_decode_tma<<<grid, kDecWarps * 32, smem, st>>>(ix, l0, l1, out_base0, out, seg0, nsegs, tk, err);
    return (int)cudaGetLastError();
}

}  // namespace excl
