// Index build on the device for the ParaPFD, LRC, LRCSeg, SegLRC, HS_SegLRC
// and HS_ParaPFD formats: hash partition, regression fits, residuals and
// minima, d-gaps and medians, and the ParaPFD blocks, with the same bytes as
// the host build (codec.cpp), which restates the reference encoders
// (ParaPFor.cpp:31-94, ParaPFD_Compression/main.cpp:163-189,
// SegLRC_Generator.cu:190-331, LRC_Generator.cu:155-287,
// LRCSeg_Generator.cu:160-215, HS_SegLRC_Generator.cu:180-594).
//
//   k_hs_shift       one thread per list: the bucket shift (from the list
//                    length and last docID, or the top k bits) and the
//                    number of buckets.
//   k_hs_offsets     one warp per list: each bucket's first element (a lower
//                    bound per bucket).
//   k_fit_segments   one thread per segment: the least-squares fit in double
//                    precision, summed in element order as the reference's
//                    host code does, every operation an explicitly rounded
//                    intrinsic so nothing is fused; then the window ranges L/R
//                    in single precision.
//   k_fit_lists      one thread per list: the same fit over the whole list
//                    (LRCSeg's residual basis, SegLRC's list-level regression),
//                    or LRC's fit in double precision.
//   k_lrc_min        one warp per segment: LRC residuals, the list minimum by
//                    atomicMin.
//   k_block_plan     one warp per segment (any length): the values to pack,
//                    the bit width (findBestB: smallest b whose exception
//                    count passes the FRAC test in single precision), the
//                    exceptions in element order, the block size.
//   k_block_pack     one warp per segment: the block at its word offset; each
//                    lane assembles whole output words (LSB-first packing).
// Block offsets come from a scan of the block sizes in between. The segment
// table, hash directory and tile map are assembled on the host from the
// bucket offsets (a few bytes per bucket).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "excl_device.cuh"
#include "runtime.h"

namespace excl {
namespace {

struct FitOut {
    float a, b;
    uint32_t L, R;
};

__device__ __forceinline__ uint32_t nbits_d(uint32_t v) { return v ? 32u - (uint32_t)__clz(v) : 0u; }

// The reference host fit (SegLRC_Generator.cu:264-331) over y[0..n).
__device__ FitOut fit_seq(const uint32_t *__restrict__ y, uint32_t n) {
    FitOut f{1.0f, 0.0f, 0u, 0u};
    if (n == 0) return f;
    if (n == 1) {
        f.b = __uint2float_rn(y[0]);
        return f;
    }
    double mx = 0.0, my = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        mx = __dadd_rn(mx, (double)i);
        my = __dadd_rn(my, (double)y[i]);
    }
    mx = __ddiv_rn(mx, (double)n);
    my = __ddiv_rn(my, (double)n);
    double sxx = 0.0, sxy = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        const double dx = __dsub_rn((double)i, mx);
        sxx = __dadd_rn(sxx, __dmul_rn(dx, dx));
        sxy = __dadd_rn(sxy, __dmul_rn(dx, __dsub_rn((double)y[i], my)));
    }
    f.a = __double2float_rn(__ddiv_rn(sxy, sxx));
    f.b = __double2float_rn(__dsub_rn(my, __dmul_rn((double)f.a, mx)));
    float left = 0.0f, right = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
        const float d = __fsub_rn(__fdiv_rn(__fsub_rn(__uint2float_rn(y[i]), f.b), f.a), __uint2float_rn(i));
        if (d > left) left = d;
        else if (d < right) right = d;
    }
    f.L = __float2uint_rz(left) + 1u;
    f.R = __float2uint_rz(__fsub_rn(0.0f, right)) + 1u;
    return f;
}

// double -> int32 as the host build's conversion gives it on x86-64
// (cvttsd2si): truncation, and 0x80000000 for NaN or out of range.
__device__ __forceinline__ int32_t d2i_host(double v) {
    if (!(v > -2147483649.0 && v < 2147483648.0)) return (int32_t)0x80000000u;
    return __double2int_rz(v);
}

// The reference's LRC fit (LRC_Generator.cu:221-287) over y[0..n), in the
// SegReg slots: a = slope, b = the intercept's bits, L = the range's bits.
__device__ SegReg fit_lrc_seq(const uint32_t *__restrict__ y, uint32_t n) {
    float slope = 1.0f, range = 0.0f;
    int32_t icpt = 0;
    if (n == 1) icpt = (int32_t)y[0];
    if (n > 1) {
        double mx = 0.0, my = 0.0;
        for (uint32_t i = 0; i < n; ++i) {
            mx = __dadd_rn(mx, (double)i);
            my = __dadd_rn(my, (double)y[i]);
        }
        mx = __ddiv_rn(mx, (double)n);
        my = __ddiv_rn(my, (double)n);
        double sxx = 0.0, sxy = 0.0;
        for (uint32_t i = 0; i < n; ++i) {
            const double dx = __dsub_rn((double)i, mx);
            sxx = __dadd_rn(sxx, __dmul_rn(dx, dx));
            sxy = __dadd_rn(sxy, __dmul_rn(dx, __dsub_rn((double)y[i], my)));
        }
        const double s = __ddiv_rn(sxy, sxx), c = __dsub_rn(my, __dmul_rn(s, mx));
        double left = 0.0, right = 0.0;
        for (uint32_t i = 0; i < n; ++i) {
            const double d = __dsub_rn(__ddiv_rn(__dsub_rn((double)y[i], c), s), (double)i);
            if (d > left) left = d;
            else if (d < right) right = d;
        }
        slope = __double2float_rn(s);
        icpt = d2i_host(c);
        range = __double2float_rn(__dsub_rn(left, right));
    }
    return SegReg{slope, __int_as_float(icpt), __float_as_uint(range), 0u};
}

struct SegTab {
    const uint32_t *seg_list;   // list of each segment
    const uint32_t *seg_start;  // first element within its list
    const uint32_t *seg_count;
    const uint64_t *list_off;   // CSR offsets of the lists in docs
};

__global__ void k_fit_segments(const uint32_t *__restrict__ docs, SegTab t, uint32_t nsegs, SegReg *__restrict__ reg) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nsegs) return;
    const uint32_t *y = docs + t.list_off[t.seg_list[g]] + t.seg_start[g];
    const FitOut f = fit_seq(y, t.seg_count[g]);
    reg[g] = SegReg{f.a, f.b, f.L, f.R};
}

// Lists longer than kHostFit postings are fitted on host threads instead: a
// sequential double-precision sum runs ~30x faster on a CPU core than on one
// GPU thread, and the fit must be sequential to keep the reference's rounding.
constexpr uint32_t kHostFit = 1u << 16;

__global__ void k_fit_lists(const uint32_t *__restrict__ docs, const uint64_t *__restrict__ list_off, uint32_t nlists,
                            bool lrc, SegReg *__restrict__ lreg) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlists) return;
    const uint64_t o = list_off[l];
    const uint32_t n = (uint32_t)(list_off[l + 1] - o);
    if (n > kHostFit) return;
    if (lrc) {
        lreg[l] = fit_lrc_seq(docs + o, n);
    } else {
        const FitOut f = fit_seq(docs + o, n);
        lreg[l] = SegReg{f.a, f.b, f.L, f.R};
    }
}

// HS partition (HS_SegLRC_Generator.cu:545-581): the shift from the expected
// bucket size, or the top kbits of a ubits-bit universe.
__global__ void k_hs_shift(const uint32_t *__restrict__ docs, const uint64_t *__restrict__ list_off, uint32_t nlists,
                           uint32_t bucket, uint32_t kbits, uint32_t ubits, uint32_t *__restrict__ shift,
                           uint32_t *__restrict__ nbk) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlists) return;
    const uint64_t o = list_off[l];
    const uint32_t n = (uint32_t)(list_off[l + 1] - o), last = docs[o + n - 1];
    const uint32_t maxb = nbits_d(last);
    uint32_t s;
    if (kbits) s = ubits > kbits ? ubits - kbits : 0u;
    else if (n <= bucket) s = maxb;
    else s = maxb - nbits_d((n + bucket - 1) / bucket);
    shift[l] = s;
    const uint64_t nb = (s >= 32 ? 0ull : ((uint64_t)last >> s)) + 1u;
    nbk[l] = nb >= 0xffffffffull ? 0xffffffffu : (uint32_t)nb;
}

// off[base[l] + b] = first element of list l whose docID >> shift >= b, for
// b in [0, nb); off[base[l] + nb] = n.
__global__ void k_hs_offsets(const uint32_t *__restrict__ docs, const uint64_t *__restrict__ list_off, uint32_t nlists,
                             const uint32_t *__restrict__ shift, const uint32_t *__restrict__ nbk,
                             const uint64_t *__restrict__ base, uint32_t *__restrict__ off) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t l = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (l >= nlists) return;
    const uint64_t o = list_off[l];
    const uint32_t n = (uint32_t)(list_off[l + 1] - o), s = shift[l], nb = nbk[l];
    const uint32_t *y = docs + o;
    uint32_t *out = off + base[l];
    for (uint32_t b = lane; b <= nb; b += 32) {
        if (b == nb) {
            out[b] = n;
            continue;
        }
        const uint64_t key = s >= 32 ? 0ull : (uint64_t)b << s;
        uint32_t lo = 0, hi = n;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if ((uint64_t)y[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        out[b] = lo;
    }
}

constexpr int kBuildWarps = 8;
constexpr uint32_t kErrBuildFormat = 1u;  // a block not representable (b = 32) or a residual spread > 31 bits
constexpr uint32_t kErrBuildOrder = 2u;   // a list is not strictly increasing

// LRC prediction (LRC_Generator_kernel.cu:70): (int)((float)i * slope) + icpt.
__device__ __forceinline__ uint32_t lrc_pred(uint32_t i, float slope, int32_t icpt) {
    return (uint32_t)__float2int_rz(__fmul_rn(__int2float_rn((int32_t)i), slope)) + (uint32_t)icpt;
}

// LRC's residual minimum over each list (LRC_Generator.cu:165-177).
__global__ void __launch_bounds__(kBuildWarps * 32) k_lrc_min(const uint32_t *__restrict__ docs, SegTab t,
                                                              uint32_t nsegs, const SegReg *__restrict__ lreg,
                                                              int32_t *__restrict__ lmin) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t g = blockIdx.x * kBuildWarps + (threadIdx.x >> 5);
    if (g >= nsegs) return;
    const uint32_t l = t.seg_list[g];
    const uint32_t s0 = t.seg_start[g], n = t.seg_count[g];
    const uint32_t *y = docs + t.list_off[l] + s0;
    const SegReg f = lreg[l];
    int32_t mn = INT_MAX;
    for (uint32_t i = lane; i < n; i += 32)
        mn = min(mn, (int32_t)(y[i] - lrc_pred(s0 + i, f.a, __float_as_int(f.b))));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    if (lane == 0) atomicMin(lmin + l, mn);
}

struct Plan {
    uint32_t lb, eb, hb, en;  // block parameters (NewPFD: eb = the Simple-16 stream's words, hb unused)
    uint32_t words;           // block size
};

// Value k of a NewPFD block's exception stream (NewPFor.cpp:91-106): the en
// position codes (the first position, then gaps minus one), then the en high
// parts, from the exceptions in element order.
__device__ __forceinline__ uint32_t newpfd_stream_value(const uint32_t *xp, const uint32_t *xh, uint32_t en,
                                                        uint32_t k) {
    if (k >= en) return xh[k - en];
    return k ? xp[k] - xp[k - 1] - 1u : xp[0];
}

// Width of value j of Simple-16 layout k.
__device__ __forceinline__ uint32_t s16_width(uint32_t k, uint32_t j) {
    const uint32_t c0 = kS16Dev[k][0], c1 = kS16Dev[k][2];
    return j < c0 ? kS16Dev[k][1] : (j < c0 + c1 ? kS16Dev[k][3] : kS16Dev[k][5]);
}

// The Simple-16 packing of a NewPFD block's exception stream, warp-parallel
// over the layouts: for each word, lane k < 16 tests layout k on the next
// values and the first layout (in table order) that holds them is taken, as
// the sequential encoder takes it (NewPFor.cpp, Simple16.h). Writes the words
// to `out` and returns their count, or ~0u when a value needs more than 28
// bits. Every lane of the warp calls it.
__device__ uint32_t s16_pack_warp(const uint32_t *xp, const uint32_t *xh, uint32_t en, uint32_t *out, uint32_t lane) {
    const uint32_t V = 2u * en;
    uint32_t i = 0, nw = 0;
    while (i < V) {
        bool fits = false;
        uint32_t vol = 0;
        if (lane < 16u) {
            const uint32_t total = (uint32_t)kS16Dev[lane][0] + kS16Dev[lane][2] + kS16Dev[lane][4];
            vol = min(total, V - i);
            fits = true;
            for (uint32_t j = 0; j < vol && fits; ++j)
                fits = newpfd_stream_value(xp, xh, en, i + j) < (1u << s16_width(lane, j));
        }
        const uint32_t m = __ballot_sync(0xffffffffu, fits);
        if (!m) return ~0u;
        const uint32_t k = (uint32_t)(__ffs(m) - 1);
        if (lane == k) {
            uint32_t wv = k << 28, sh = 0;
            for (uint32_t j = 0; j < vol; ++j) {
                wv |= newpfd_stream_value(xp, xh, en, i + j) << sh;
                sh += s16_width(k, j);
            }
            out[nw] = wv;
        }
        i += __shfl_sync(0xffffffffu, vol, k);
        ++nw;
    }
    return nw;
}

// One warp per segment of any length. vals (per element) receives the values
// to pack; ex_pos / ex_high (per element, in the segment's own range) its
// exceptions in element order.
__global__ void __launch_bounds__(kBuildWarps * 32) k_block_plan(const uint32_t *__restrict__ docs, SegTab t,
                                                                 uint32_t nsegs, uint32_t codec, float frac,
                                                                 const SegReg *__restrict__ reg,
                                                                 const SegReg *__restrict__ lreg,
                                                                 const int32_t *__restrict__ lmin,
                                                                 uint32_t *__restrict__ vals,
                                                                 uint32_t *__restrict__ ex_pos,
                                                                 uint32_t *__restrict__ ex_high,
                                                                 uint32_t *__restrict__ head, uint32_t *__restrict__ aux,
                                                                 Plan *__restrict__ plan, uint32_t *__restrict__ s16w,
                                                                 uint32_t *__restrict__ err) {
    __shared__ uint32_t s_hist[kBuildWarps][33];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t g = blockIdx.x * kBuildWarps + w;
    if (g >= nsegs) return;
    const uint32_t l = t.seg_list[g];
    const uint64_t lo = t.list_off[l];
    const uint32_t s0 = t.seg_start[g], n = t.seg_count[g];
    const uint32_t *y = docs + lo + s0;
    uint32_t *out = vals + lo + s0;
    uint32_t *xp = ex_pos + lo + s0, *xh = ex_high + lo + s0;
    const bool dgap = codec_is_dgap(codec);
    const bool seg_fit = codec == EXCL_CODEC_SEGLRC || codec == EXCL_CODEC_HS_SEGLRC;
    const SegReg f = dgap ? SegReg{1.0f, 0.0f, 0u, 0u} : (seg_fit ? reg[g] : lreg[l]);
    if (lane < 32) s_hist[w][lane] = 0;
    if (lane == 0) s_hist[w][32] = 0;
    // pass 1: strict order; d-gaps (across the whole list) or residuals
    bool unordered = false;
    int32_t mn = INT_MAX;
    for (uint32_t i = lane; i < n; i += 32) {
        const uint32_t yi = y[i];
        const bool first = s0 + i == 0;
        unordered |= !first && yi <= y[(int)i - 1];
        if (dgap) {
            out[i] = first ? yi : yi - y[(int)i - 1];
        } else {
            int32_t r;
            if (codec == EXCL_CODEC_LRC) {
                r = (int32_t)(yi - lrc_pred(s0 + i, f.a, __float_as_int(f.b)));
            } else {
                // LRCSeg: list-level index and fit; SegLRC / HS_SegLRC: segment-local
                const uint32_t idx = codec == EXCL_CODEC_LRCSEG ? s0 + i : i;
                r = (int32_t)(yi - (uint32_t)__float2int_rz(__fmaf_rn(__uint2float_rn(idx), f.a, f.b)));
            }
            out[i] = (uint32_t)r;
            mn = min(mn, r);
        }
    }
    if (__any_sync(0xffffffffu, unordered) && lane == 0) atomicOr(err, kErrBuildOrder);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    if (codec == EXCL_CODEC_LRC) mn = lmin[l];
    __syncwarp();
    // pass 2: residuals minus the minimum; histogram of the value widths
    // (lanes with the same width add once)
    bool bad = false;
    for (uint32_t c0 = 0; c0 < n; c0 += 32) {
        const uint32_t i = c0 + lane;
        uint32_t bin = 33u;
        if (i < n) {
            uint32_t v = out[i];
            if (!dgap) {
                const int64_t d = (int64_t)(int32_t)v - mn;
                bad |= d > 0x7fffffffLL;
                v = (uint32_t)d;
                out[i] = v;
            }
            bin = nbits_d(v);
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, bin);
        if (bin < 33u && lane == (uint32_t)(__ffs(peers) - 1)) s_hist[w][bin] += __popc(peers);
        __syncwarp();
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(err, kErrBuildFormat);
    if (lane == 0) {
        head[g] = y[0];
        aux[g] = dgap ? y[n / 2] : (codec == EXCL_CODEC_LRC ? 0u : (uint32_t)mn);
    }
    __syncwarp();
    // findBestB (ParaPFor.cpp:31-53): the smallest width b (lane b) whose
    // count of wider values passes the FRAC test in single precision
    const float lim = __fmul_rn(frac, __uint2float_rn(n));
    uint32_t above = 0;
    for (uint32_t k = lane + 1; k <= 32; ++k) above += s_hist[w][k];
    const uint32_t okm = __ballot_sync(0xffffffffu, __uint2float_rn(above) <= lim);
    const uint32_t lb = okm ? (uint32_t)(__ffs(okm) - 1) : 32u;
    Plan p{lb, 0u, 0u, 0u, 0u};
    if (lb >= 32) {
        if (lane == 0) atomicOr(err, kErrBuildFormat);
        p.lb = 0;
    } else {
        // exceptions in element order
        uint32_t en = 0, orh = 0, last = 0;
        for (uint32_t c0 = 0; c0 < n; c0 += 32) {
            const uint32_t i = c0 + lane;
            const uint32_t v = i < n ? out[i] : 0u;
            const bool ex = i < n && nbits_d(v) > lb;
            const uint32_t m = __ballot_sync(0xffffffffu, ex);
            if (ex) {
                const uint32_t k = en + __popc(m & ((1u << lane) - 1u));
                xp[k] = i;
                xh[k] = v >> lb;
                orh |= v >> lb;
            }
            if (m) last = c0 + 31u - __clz(m);
            en += __popc(m);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) orh |= __shfl_xor_sync(0xffffffffu, orh, o);
        p.en = en;
        if (en && codec == EXCL_CODEC_NEWPFD) {
            // NewPFD: the exceptions go to one Simple-16 stream, packed here
            // into the segment's scratch slot (2 words per element is enough)
            __syncwarp();  // the exception lists are written
            const uint32_t nw = en > 0xffffu ? ~0u : s16_pack_warp(xp, xh, en, s16w + 2 * (lo + s0), lane);
            if (nw == ~0u) {
                if (lane == 0) atomicOr(err, kErrBuildFormat);
                p.en = 0;
            } else {
                p.eb = nw;
            }
        } else if (en) {
            p.eb = nbits_d(last);
            p.hb = nbits_d(orh);
            // not representable in the descriptor (ParaPFor.cpp:79-88: eb from the last position, hb from the highs, 5-bit fields)
            if (p.eb >= 32 || p.hb >= 32 || en > 0xffffu) {
                if (lane == 0) atomicOr(err, kErrBuildFormat);
                p.en = p.eb = p.hb = 0;
            }
        }
    }
    p.words = 1u + (uint32_t)(((uint64_t)n * p.lb + 31u) >> 5);
    if (p.en && codec == EXCL_CODEC_NEWPFD) p.words += p.eb;
    else if (p.en)
        p.words += (uint32_t)(((uint64_t)p.en * p.eb + 31u) >> 5) + (uint32_t)(((uint64_t)p.en * p.hb + 31u) >> 5);
    if (lane == 0) plan[g] = p;
}

// Word k of an LSB-first packing of (src[i] & mask), i in [0, n), at `bits` bits per value.
__device__ __forceinline__ uint32_t packed_word(const uint32_t *src, uint32_t n, uint32_t bits, uint32_t mask,
                                                uint32_t k) {
    const uint64_t b0 = (uint64_t)k * 32u;
    const uint64_t last = (b0 + 31u) / bits + 1u;
    const uint32_t i0 = (uint32_t)(b0 / bits), i1 = (uint32_t)(last < n ? last : n);
    uint32_t w = 0;
    for (uint32_t i = i0; i < i1; ++i) {
        const int64_t sh = (int64_t)i * bits - (int64_t)b0;  // position of value i's bit 0 in this word
        const uint64_t val = src[i] & mask;
        if (sh >= 0) w |= (uint32_t)(val << sh);
        else w |= (uint32_t)(val >> (-sh));
    }
    return w;
}

__global__ void __launch_bounds__(kBuildWarps * 32) k_block_pack(const uint32_t *__restrict__ vals,
                                                                 const uint32_t *__restrict__ ex_pos,
                                                                 const uint32_t *__restrict__ ex_high, SegTab t,
                                                                 uint32_t nsegs, const Plan *__restrict__ plan,
                                                                 const uint64_t *__restrict__ gword,
                                                                 const uint32_t *__restrict__ s16w, uint32_t codec,
                                                                 uint32_t *__restrict__ words) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t g = blockIdx.x * kBuildWarps + (threadIdx.x >> 5);
    if (g >= nsegs) return;
    const Plan p = plan[g];
    const uint32_t n = t.seg_count[g];
    const uint64_t e0 = t.list_off[t.seg_list[g]] + t.seg_start[g];
    uint32_t *blk = words + gword[g];
    const uint32_t wl = (uint32_t)(((uint64_t)n * p.lb + 31u) >> 5);
    const bool npfd = codec == EXCL_CODEC_NEWPFD;
    // descriptors: ParaPFor.cpp:88-91; NewPFD b << 26 | en (NewPFor.cpp:52-139)
    if (lane == 0) blk[0] = p.en ? (npfd ? (p.lb << 26) + p.en : (p.lb << 26) + (p.eb << 21) + (p.hb << 16) + p.en)
                                 : (p.lb << 26);
    if (p.lb) {
        const uint32_t mask = (1u << p.lb) - 1u;  // lb <= 31
        for (uint32_t k = lane; k < wl; k += 32) blk[1 + k] = packed_word(vals + e0, n, p.lb, mask, k);
    }
    if (p.en && npfd) {
        const uint32_t *src = s16w + 2 * e0;
        for (uint32_t k = lane; k < p.eb; k += 32) blk[1 + wl + k] = src[k];
    } else if (p.en) {
        const uint32_t we = (uint32_t)(((uint64_t)p.en * p.eb + 31u) >> 5);
        const uint32_t wh = (uint32_t)(((uint64_t)p.en * p.hb + 31u) >> 5);
        if (p.eb)
            for (uint32_t k = lane; k < we; k += 32)
                blk[1 + wl + k] = packed_word(ex_pos + e0, p.en, p.eb, 0xffffffffu, k);
        if (p.hb)
            for (uint32_t k = lane; k < wh; k += 32)
                blk[1 + wl + we + k] = packed_word(ex_high + e0, p.en, p.hb, 0xffffffffu, k);
    }
}

__global__ void k_gather_last(const uint32_t *__restrict__ docs, const uint64_t *__restrict__ list_off, uint32_t nlists,
                              uint32_t *__restrict__ last) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < nlists) last[l] = docs[list_off[l + 1] - 1];
}

// Device buffers of one build, freed together.
struct Scratch {
    std::vector<void *> p;
    template <class T>
    bool get(T **x, size_t count) {
        *x = nullptr;
        if (cudaMalloc(reinterpret_cast<void **>(x), std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            *x = nullptr;
            return false;
        }
        p.push_back(*x);
        return true;
    }
    ~Scratch() {
        for (void *x : p) cudaFree(x);
    }
};

bool device_codec(uint32_t c) {
    return c == EXCL_CODEC_PARAPFD || c == EXCL_CODEC_SEGLRC || c == EXCL_CODEC_LRC || c == EXCL_CODEC_LRCSEG ||
           c == EXCL_CODEC_HS_SEGLRC || c == EXCL_CODEC_HS_PARAPFD || c == EXCL_CODEC_NEWPFD;
}

}  // namespace
}  // namespace excl

using namespace excl;

extern "C" int excl_index_build_device(excl_ctx *ctx, const uint32_t *d_docs, const uint64_t *list_offsets,
                                       uint32_t nlists, const excl_build_params *p, excl_index **out) {
    if (!ctx || !d_docs || !list_offsets || !p || !out || nlists == 0) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    *out = nullptr;
    const uint32_t B = p->block, codec = p->codec;
    if (p->codecs || !device_codec(codec)) return EXCL_E_INVALID;
    if (B < kMinBlock || B > kTileKeys || (B & (B - 1))) return EXCL_E_INVALID;
    const bool hs = codec_is_hs(codec);
    if (hs && !p->hs_kbits && p->hs_bucket == 0) return EXCL_E_INVALID;
    for (uint32_t l = 0; l < nlists; ++l)
        if (list_offsets[l + 1] <= list_offsets[l] || list_offsets[l + 1] - list_offsets[l] > 0xffffffffull)
            return EXCL_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    Scratch sc;
    // offsets relative to the first list, so d_docs may start anywhere
    std::vector<uint64_t> loff(nlists + 1);
    for (uint32_t l = 0; l <= nlists; ++l) loff[l] = list_offsets[l] - list_offsets[0];
    const uint64_t npost = loff[nlists];
    const uint32_t *docs0 = d_docs + list_offsets[0];  // the kernels index from the first list
    uint64_t *d_loff = nullptr;
    uint32_t *d_err = nullptr;
    if (!sc.get(&d_loff, (size_t)nlists + 1) || !sc.get(&d_err, 1)) return EXCL_E_NOMEM;
    cudaError_t e = cudaMemcpyAsync(d_loff, loff.data(), loff.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, 4, st);

    // segment table (host): fixed blocks, or the hash buckets (cut into
    // blocks for HS_ParaPFD) from the bucket offsets computed on the device
    std::vector<uint32_t> seg_list, seg_start, seg_count, seg_base(nlists), nseg(nlists);
    std::vector<uint32_t> hshift(nlists), hnb(nlists), boff;
    std::vector<uint64_t> bbase(nlists + 1, 0);
    if (e == cudaSuccess && hs) {
        uint32_t *d_shift = nullptr, *d_nb = nullptr;
        if (!sc.get(&d_shift, nlists) || !sc.get(&d_nb, nlists)) return EXCL_E_NOMEM;
        k_hs_shift<<<(nlists + 127) / 128, 128, 0, st>>>(docs0, d_loff, nlists, p->hs_bucket, p->hs_kbits,
                                                         p->hs_ubits, d_shift, d_nb);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(hshift.data(), d_shift, (size_t)nlists * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hnb.data(), d_nb, (size_t)nlists * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        for (uint32_t l = 0; e == cudaSuccess && l < nlists; ++l) {
            if (hnb[l] == 0xffffffffu) {
                ctx_error(ctx, "list %u: too many hash buckets", l);
                return EXCL_E_FORMAT;
            }
            bbase[l + 1] = bbase[l] + hnb[l] + 1;
        }
        uint32_t *d_boff = nullptr;
        uint64_t *d_bbase = nullptr;
        if (e == cudaSuccess && (!sc.get(&d_boff, bbase[nlists]) || !sc.get(&d_bbase, (size_t)nlists + 1)))
            return EXCL_E_NOMEM;
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_bbase, bbase.data(), bbase.size() * 8, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            k_hs_offsets<<<(nlists + 7) / 8, 256, 0, st>>>(docs0, d_loff, nlists, d_shift, d_nb, d_bbase, d_boff);
            e = cudaGetLastError();
        }
        boff.resize(bbase[nlists]);
        if (e == cudaSuccess) e = cudaMemcpyAsync(boff.data(), d_boff, boff.size() * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    std::vector<uint32_t> bfirst;  // per list: bucket -> first segment within the list (nb + 1 each)
    for (uint32_t l = 0; e == cudaSuccess && l < nlists; ++l) {
        const uint32_t n = (uint32_t)(loff[l + 1] - loff[l]);
        seg_base[l] = (uint32_t)seg_list.size();
        if (!hs) {
            for (uint32_t s0 = 0; s0 < n; s0 += B) {
                seg_list.push_back(l);
                seg_start.push_back(s0);
                seg_count.push_back(std::min(B, n - s0));
            }
        } else {
            const uint32_t *o = boff.data() + bbase[l];
            const uint32_t cut = codec == EXCL_CODEC_HS_PARAPFD ? B : 0xffffffffu;
            for (uint32_t b = 0; b < hnb[l]; ++b) {
                bfirst.push_back((uint32_t)seg_list.size() - seg_base[l]);
                for (uint32_t k = o[b]; k < o[b + 1]; k += std::min(cut, o[b + 1] - k)) {
                    seg_list.push_back(l);
                    seg_start.push_back(k);
                    seg_count.push_back(std::min(cut, o[b + 1] - k));
                }
            }
            bfirst.push_back((uint32_t)seg_list.size() - seg_base[l]);
        }
        nseg[l] = (uint32_t)seg_list.size() - seg_base[l];
    }
    if (e != cudaSuccess) return cuda_status(ctx, e, "device build");
    if (seg_list.size() > 0xffffffffull) return EXCL_E_CAPACITY;
    const uint32_t ns = (uint32_t)seg_list.size();

    uint32_t *d_slist = nullptr, *d_sstart = nullptr, *d_scount = nullptr, *d_vals = nullptr, *d_xpos = nullptr,
             *d_xhigh = nullptr, *d_head = nullptr, *d_aux = nullptr, *d_words = nullptr;
    uint64_t *d_gword = nullptr;
    SegReg *d_reg = nullptr, *d_lreg = nullptr;
    int32_t *d_lmin = nullptr;
    Plan *d_plan = nullptr;
    if (!sc.get(&d_slist, ns) || !sc.get(&d_sstart, ns) || !sc.get(&d_scount, ns) || !sc.get(&d_head, ns) ||
        !sc.get(&d_aux, ns) || !sc.get(&d_reg, ns) || !sc.get(&d_plan, ns) || !sc.get(&d_gword, (size_t)ns + 1) ||
        !sc.get(&d_lreg, nlists) || !sc.get(&d_lmin, nlists) || !sc.get(&d_vals, npost) ||
        !sc.get(&d_xpos, npost) || !sc.get(&d_xhigh, npost))
        return EXCL_E_NOMEM;
    uint32_t *d_s16 = nullptr;  // NewPFD: each segment's Simple-16 exception stream, 2 words per element
    if (codec == EXCL_CODEC_NEWPFD && !sc.get(&d_s16, 2 * npost)) return EXCL_E_NOMEM;
    const std::vector<int32_t> lmin_init(nlists, INT_MAX);
    e = cudaMemcpyAsync(d_slist, seg_list.data(), (size_t)ns * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_sstart, seg_start.data(), (size_t)ns * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_scount, seg_count.data(), (size_t)ns * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_lmin, lmin_init.data(), (size_t)nlists * 4, cudaMemcpyHostToDevice, st);
    const SegTab t{d_slist, d_sstart, d_scount, d_loff};

    // list-level fits: on the device for short lists; long lists are copied to
    // the host (pinned) and fitted by host threads. LRC and LRCSeg residuals
    // need them, so those builds wait; SegLRC and HS_SegLRC only store them.
    const bool lrc = codec == EXCL_CODEC_LRC;
    const bool list_fit = !codec_is_dgap(codec);
    const bool fit_first = lrc || codec == EXCL_CODEC_LRCSEG;
    std::vector<uint32_t> host_fit;
    uint64_t host_words = 0;
    if (list_fit)
        for (uint32_t l = 0; l < nlists; ++l)
            if (loff[l + 1] - loff[l] > kHostFit) {
                host_fit.push_back(l);
                host_words += loff[l + 1] - loff[l];
            }
    uint32_t *h_long = nullptr;
    cudaEvent_t long_ready = nullptr;
    std::vector<SegReg> host_reg(host_fit.size());
    std::thread fitter;
    auto join_fitter = [&]() {
        if (fitter.joinable()) fitter.join();
        if (long_ready) cudaEventDestroy(long_ready);
        long_ready = nullptr;
        if (h_long) cudaFreeHost(h_long);
        h_long = nullptr;
    };
    if (e == cudaSuccess && list_fit) {
        k_fit_lists<<<(nlists + 127) / 128, 128, 0, st>>>(docs0, d_loff, nlists, lrc, d_lreg);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && !host_fit.empty()) {
        e = cudaMallocHost((void **)&h_long, host_words * 4);
        uint64_t o = 0;
        for (uint32_t l : host_fit) {
            const uint64_t n = loff[l + 1] - loff[l];
            if (e == cudaSuccess) e = cudaMemcpyAsync(h_long + o, docs0 + loff[l], n * 4, cudaMemcpyDeviceToHost, st);
            o += n;
        }
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&long_ready, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(long_ready, st);
        if (e == cudaSuccess)
            fitter = std::thread([&]() {
                if (cudaEventSynchronize(long_ready) != cudaSuccess) return;
                std::vector<uint64_t> base(host_fit.size() + 1, 0);
                for (size_t i = 0; i < host_fit.size(); ++i)
                    base[i + 1] = base[i] + (loff[host_fit[i] + 1] - loff[host_fit[i]]);
                std::atomic<size_t> next{0};
                const unsigned nth = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(),
                                                                      (unsigned)host_fit.size()));
                std::vector<std::thread> pool;
                for (unsigned k = 0; k < nth; ++k)
                    pool.emplace_back([&]() {
                        for (size_t i; (i = next.fetch_add(1)) < host_fit.size();) {
                            const uint32_t *y = h_long + base[i];
                            const uint32_t n = (uint32_t)(base[i + 1] - base[i]);
                            if (lrc) {
                                SegReg r{};
                                int32_t c;
                                float range;
                                fit_lrc_host(y, n, &r.a, &c, &range);
                                std::memcpy(&r.b, &c, 4);
                                std::memcpy(&r.L, &range, 4);
                                host_reg[i] = r;
                            } else {
                                host_reg[i] = fit_host(y, n);
                            }
                        }
                    });
                for (auto &th : pool) th.join();
            });
    }
    if (e == cudaSuccess && fit_first && !host_fit.empty()) {
        // the residuals need every list fit on the device first
        join_fitter();
        for (size_t i = 0; i < host_fit.size() && e == cudaSuccess; ++i)
            e = cudaMemcpyAsync(d_lreg + host_fit[i], &host_reg[i], sizeof(SegReg), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host_reg is pageable: let the copies finish
    }
    if (e == cudaSuccess && (codec == EXCL_CODEC_SEGLRC || codec == EXCL_CODEC_HS_SEGLRC)) {
        k_fit_segments<<<(ns + 127) / 128, 128, 0, st>>>(docs0, t, ns, d_reg);
        e = cudaGetLastError();
    }
    const uint32_t pgrid = (ns + kBuildWarps - 1) / kBuildWarps;
    if (e == cudaSuccess && lrc) {
        k_lrc_min<<<pgrid, kBuildWarps * 32, 0, st>>>(docs0, t, ns, d_lreg, d_lmin);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_block_plan<<<pgrid, kBuildWarps * 32, 0, st>>>(docs0, t, ns, codec, p->frac, d_reg, d_lreg, d_lmin, d_vals,
                                                         d_xpos, d_xhigh, d_head, d_aux, d_plan, d_s16, d_err);
        e = cudaGetLastError();
    }
    // block offsets: a scan of the block sizes (host; 20 bytes per segment)
    std::vector<Plan> plan(ns);
    uint32_t flags = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(plan.data(), d_plan, (size_t)ns * sizeof(Plan), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flags, d_err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess || flags) {
        join_fitter();
        if (e != cudaSuccess) return cuda_status(ctx, e, "device build");
        if (flags & kErrBuildOrder) {
            ctx_error(ctx, "posting lists are not strictly increasing");
            return EXCL_E_INVALID;
        }
        ctx_error(ctx, "a block is not representable (ParaPFD or NewPFD limits) or a residual spread exceeds 31 bits");
        return EXCL_E_FORMAT;
    }
    std::vector<uint64_t> gword(ns + 1, 0);
    for (uint32_t g = 0; g < ns; ++g) gword[g + 1] = gword[g] + plan[g].words;
    if (!sc.get(&d_words, gword[ns] + kWordPad)) {
        join_fitter();
        return EXCL_E_NOMEM;
    }
    e = cudaMemcpyAsync(d_gword, gword.data(), gword.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_words, 0, (gword[ns] + kWordPad) * 4, st);
    if (e == cudaSuccess) {
        k_block_pack<<<pgrid, kBuildWarps * 32, 0, st>>>(d_vals, d_xpos, d_xhigh, t, ns, d_plan, d_gword, d_s16, codec,
                                                         d_words);
        e = cudaGetLastError();
    }
    // the host image
    excl_index *ix = new (std::nothrow) excl_index();
    if (!ix) {
        join_fitter();
        return EXCL_E_NOMEM;
    }
    ix->nlists = nlists;
    ix->lists.resize(nlists);
    ix->words.resize(gword[ns] + kWordPad);
    ix->seg_head.resize(ns);
    ix->seg_rec.resize(ns);
    ix->seg_reg.assign(ns, SegReg{1.0f, 0.0f, 0, 0});
    std::vector<uint32_t> aux(ns), last(nlists);
    std::vector<SegReg> lreg(nlists);
    std::vector<int32_t> lmin(nlists);
    uint32_t *d_last = nullptr;
    if (e == cudaSuccess && !sc.get(&d_last, nlists)) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaMemcpyAsync(ix->words.data(), d_words, ix->words.size() * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ix->seg_head.data(), d_head, (size_t)ns * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(aux.data(), d_aux, (size_t)ns * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && (codec == EXCL_CODEC_SEGLRC || codec == EXCL_CODEC_HS_SEGLRC))
        e = cudaMemcpyAsync(ix->seg_reg.data(), d_reg, (size_t)ns * sizeof(SegReg), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && list_fit)
        e = cudaMemcpyAsync(lreg.data(), d_lreg, (size_t)nlists * sizeof(SegReg), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && lrc)
        e = cudaMemcpyAsync(lmin.data(), d_lmin, (size_t)nlists * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) {
        // the lists' last docIDs
        k_gather_last<<<(nlists + 255) / 256, 256, 0, st>>>(docs0, d_loff, nlists, d_last);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(last.data(), d_last, (size_t)nlists * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    join_fitter();
    if (e != cudaSuccess) {
        delete ix;
        return cuda_status(ctx, e, "device build");
    }
    for (size_t i = 0; i < host_fit.size(); ++i) lreg[host_fit[i]] = host_reg[i];
    std::vector<uint32_t> ldir;
    ix->postings = npost;
    size_t bf = 0;  // position in bfirst
    for (uint32_t l = 0; l < nlists; ++l) {
        ListDesc &d = ix->lists[l];
        d.n = (uint32_t)(loff[l + 1] - loff[l]);
        d.codec = codec;
        d.log2_block = hs ? 0u : (uint32_t)__builtin_ctz(B);
        d.seg_base = seg_base[l];
        d.nseg = nseg[l];
        d.word_base = gword[seg_base[l]];
        d.first_doc = ix->seg_head[seg_base[l]];
        d.last_doc = last[l];
        d.model = kNoModel;
        if (lrc) {
            // LRC: slope, the intercept moved by the list's residual minimum, range
            int32_t icpt;
            std::memcpy(&icpt, &lreg[l].b, 4);
            icpt = (int32_t)((uint32_t)icpt + (uint32_t)lmin[l]);
            std::memcpy(&d.reg[0], &lreg[l].a, 4);
            std::memcpy(&d.reg[1], &icpt, 4);
            d.reg[2] = lreg[l].L;
            d.reg[3] = 0;
        } else if (list_fit) {
            std::memcpy(d.reg, &lreg[l], sizeof(SegReg));
        }
        for (uint32_t s = 0; s < nseg[l]; ++s) {
            const uint32_t g = seg_base[l] + s;
            SegRec &r = ix->seg_rec[g];
            r.start = seg_start[g];
            r.off = (uint32_t)(gword[g] - d.word_base);
            r.aux = aux[g];
            r.count = seg_count[g];
        }
        d.dir_base = (uint32_t)ix->dir.size();
        d.tile_base = (uint32_t)ix->tilemap.size();
        if (hs) {
            d.dir_shift = hshift[l];
            d.ndir = hnb[l];
            ix->dir.insert(ix->dir.end(), bfirst.begin() + bf, bfirst.begin() + bf + hnb[l] + 1);
            bf += hnb[l] + 1;
            if (variable_list_tiles(seg_count.data() + seg_base[l], nseg[l], ix->tilemap)) {
                delete ix;
                ctx_error(ctx, "hash bucket larger than 2^24 postings");
                return EXCL_E_FORMAT;
            }
            d.ntiles = (uint32_t)ix->tilemap.size() - d.tile_base;
        } else {
            fixed_list_directory(d, ix->seg_head.data() + d.seg_base, d.nseg, ldir);
            ix->dir.insert(ix->dir.end(), ldir.begin(), ldir.end());
            d.ntiles = d.nseg;
        }
    }
    *out = ix;
    return EXCL_OK;
}
