// K1/K2 whole-list decode with TMA bulk staging.
//
// Each CTA owns a contiguous range of segments. Consecutive ParaPFD blocks are
// contiguous in the index's word array, so a run of up to 32 segments is one
// contiguous byte range: warp 0 plans the next run (32 segments' metadata
// loaded 32-wide, a ballot finds how many fit a 24 KB stage), and one
// cp.async.bulk copies the run into shared memory, completing on an mbarrier,
// while all warps decode the previous run from the other stage. Decoding works
// from shared memory only: bit-window extraction of each lane's run of values,
// exception patching, d-gap warp scan (ParaPFD_Decompression_kernel.cu:205-263)
// or regression reconstruction (SegLRC_Decompression_kernel.cu:249-252), then
// coalesced 128-byte stores. Hash buckets of more than 256 postings are not
// staged; their 256-slices are decoded from global memory.
//
// No multicast is used: each CTA copies only into its own shared memory.
#include <cuda_runtime.h>

#include "excl_device.cuh"
#include "kernels.h"

namespace excl {

constexpr int kDecWarps = 8;
constexpr uint32_t kStages = 2;          // ring of staged runs: one copy in flight while one is decoded
constexpr uint32_t kStageCap = 4096;     // words per stage (16 KB; a run of 32 segments needs ~3-13 KB)
constexpr int kDecCtasPerSm = 4;
constexpr uint32_t kDecChunk = 64;  // segments per work ticket
constexpr uint32_t kRunSegs = 32;
constexpr uint32_t kWaitLimit = 1u << 22;  // try_wait polls before giving up (a stage normally lands in microseconds)

struct alignas(16) RunMeta {
    uint64_t ob;       // output position of the segment's first docID
    uint32_t woff;     // descriptor word within the stage
    uint32_t count, start, aux, head, list;
    float a, b;
    uint32_t codec, r0, r1;  // the list's codec and list-level regression words
    uint32_t pad[3];
};

struct DecodeSmem {
    uint32_t stage[kStages][kStageCap + 8];
    RunMeta meta[kStages][kRunSegs];
    uint32_t vals[kDecWarps][kTileKeys];
    unsigned long long mbar[kStages];
    uint32_t run_n[kStages];       // segments in the run
    uint32_t run_big[kStages];     // 1: a single large bucket, not staged
    uint32_t run_first[kStages];   // global index of the run's first segment
    uint32_t have[kStages];        // 1: stage holds a planned run
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
        // independent loads; only the output position waits on the list id
        l = ix.seg_list[s];
        const SegRec rec = ix.seg_rec[s];
        gword = ix.seg_gword[s];
        bw = ix.seg_gword[s + 1] - gword;
        head = ldg(ix.seg_head + s);
        const SegReg rg = ix.seg_reg[s];
        count = rec.count;
        start = rec.start;
        aux = rec.aux;
        a = rg.a;
        bb = rg.b;
        ob = ix.post_base[l] - out_base0 + rec.start;
        codec = ix.lists[l].codec;
        r0 = ix.lists[l].reg[0];
        r1 = ix.lists[l].reg[1];
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
    }
    const uint64_t need_last = __shfl_sync(0xffffffffu, need, n - 1);
    if (lane == 0) {
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

// Exceptions of a staged block (ParaPFor.cpp:116-125): patch the high bits
// of the listed positions into vbuf[0, count).
__device__ __noinline__ void patch_exceptions(const uint32_t *lows, BlkHdr h, uint32_t count, uint32_t *vbuf,
                                              uint32_t lane) {
    __syncwarp();
    const uint32_t *pb = lows + words_for(count, h.lb);
    const uint32_t *hp = pb + words_for(h.en, h.eb);
    for (uint32_t x = lane; x < h.en; x += 32) {
        const uint32_t pbit = x * h.eb, hbit = x * h.hb;
        const uint32_t p = __funnelshift_r(pb[pbit >> 5], pb[(pbit >> 5) + 1], pbit & 31u) & ((1u << h.eb) - 1u);
        const uint32_t hv = __funnelshift_r(hp[hbit >> 5], hp[(hbit >> 5) + 1], hbit & 31u) & ((1u << h.hb) - 1u);
        if (p < count) vbuf[p] |= hv << h.lb;
    }
    __syncwarp();
}

// d-gap codecs: lane l owns a run of ceil(count/32) consecutive values; the
// segment head replaces value 0, then a warp scan turns gaps into docIDs
// (ParaPFD_Decompression_kernel.cu:205-263).
__device__ __noinline__ void decode_dgap_staged(const uint32_t *blk, const RunMeta &m, uint32_t *vbuf,
                                                uint32_t *__restrict__ out, uint32_t lane) {
    const BlkHdr h = blk_hdr(blk[0]);
    const uint32_t *lows = blk + 1;
    const uint32_t count = m.count;
    const uint32_t vpl = (count + 31u) >> 5;
    const uint32_t el = lane * vpl;
    const uint32_t mask = (1u << h.lb) - 1u;
    uint32_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const uint32_t bit = (el + q) * h.lb;
        const uint32_t wi = bit >> 5;
        v[q] = (q < (int)vpl && el + q < count) ? (__funnelshift_r(lows[wi], lows[wi + 1], bit & 31u) & mask) : 0u;
    }
    if (h.en) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (q < (int)vpl && el + q < count) vbuf[el + q] = v[q];
        if (codec_is_newpfd(m.codec)) {
            // NewPFD: exceptions from the Simple-16 stream, one lane
            __syncwarp();
            if (lane == 0) newpfd_patch(lows + words_for(count, h.lb), h.en, h.lb, 0, count, vbuf);
            __syncwarp();
        } else {
            patch_exceptions(lows, h, count, vbuf, lane);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (q < (int)vpl && el + q < count) v[q] = vbuf[el + q];
        __syncwarp();
    }
    if (lane == 0) v[0] = m.head;
    uint32_t run = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        run += v[q];
        v[q] = run;
    }
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t ex = incl - run;
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (q < (int)vpl && el + q < count) vbuf[el + q] = v[q] + ex;
    __syncwarp();
    uint32_t *o = out + m.ob;
    for (uint32_t i = lane; i < count; i += 32) o[i] = vbuf[i];
    __syncwarp();
}

// Residual codecs (LRC, LRCSeg, SegLRC, HS_SegLRC): no scan; lane l owns
// values l, l+32, ... so the 32 lanes read neighbouring words (no bank
// conflicts) and every value goes from its register straight into a coalesced
// 128-byte store. Reconstruction as the reference:
// LRC_Decompression_kernel.cu:254, SegLRC_Decompression_kernel.cu:252.
__device__ __forceinline__ void decode_resid_staged(const uint32_t *blk, const RunMeta &m, uint32_t *vbuf,
                                                    uint32_t *__restrict__ out, uint32_t lane) {
    const BlkHdr h = blk_hdr(blk[0]);
    const uint32_t *lows = blk + 1;
    const uint32_t count = m.count;
    const uint32_t mask = (1u << h.lb) - 1u;
    const int nqs = (int)((count + 31u) >> 5);  // 32-value steps this segment needs
    uint32_t v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if (q >= nqs) break;
        const uint32_t t = lane + 32u * q;
        const uint32_t bit = t * h.lb;
        const uint32_t wi = bit >> 5;
        v[q] = __funnelshift_r(lows[wi], lows[wi + 1], bit & 31u) & mask;  // past count: unused
    }
    if (h.en) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (q < nqs && lane + 32u * q < count) vbuf[lane + 32u * q] = v[q];
        patch_exceptions(lows, h, count, vbuf, lane);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (q < nqs && lane + 32u * q < count) v[q] = vbuf[lane + 32u * q];
        __syncwarp();
    }
    uint32_t *o = out + m.ob;
    if (m.codec == EXCL_CODEC_LRC) {
        const float slope = __uint_as_float(m.r0);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (q >= nqs) break;
            const uint32_t t = lane + 32u * q;
            if (t < count) o[t] = v[q] + pred_lrc(m.start + t, slope, (int32_t)m.r1);
        }
    } else if (m.codec == EXCL_CODEC_LRCSEG) {
        // list-level index: the float conversion of start + t as the reference's
        const float a = __uint_as_float(m.r0), b = __uint_as_float(m.r1);
        const uint32_t aux = m.aux, i0 = m.start;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (q >= nqs) break;
            const uint32_t t = lane + 32u * q;
            if (t < count) o[t] = v[q] + pred_fma(i0 + t, a, b) + aux;
        }
    } else {
        // segment-local index t < 256: float(lane) + 32q is exactly float(t)
        const float a = m.a, b = m.b, lf = (float)lane;
        const uint32_t aux = m.aux;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (q >= nqs) break;
            const uint32_t t = lane + 32u * q;
            const float tf = __fadd_rn(lf, 32.0f * (float)q);
            if (t < count) o[t] = v[q] + (uint32_t)__float2int_rz(__fmaf_rn(tf, a, b)) + aux;
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
        const uint32_t n = sm.run_n[b], big = sm.run_big[b], first = sm.run_first[b];
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
            if (!failed)
                for (uint32_t j = w; j < n; j += kDecWarps) {
                    const RunMeta &m = sm.meta[b][j];
                    if (codec_is_dgap(m.codec)) decode_dgap_staged(sm.stage[b] + m.woff, m, sm.vals[w], out, lane);
                    else decode_resid_staged(sm.stage[b] + m.woff, m, sm.vals[w], out, lane);
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
