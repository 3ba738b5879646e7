// Index build on the device for the ParaPFD and SegLRC formats (fixed
// segments): the regression fits, residuals and segment minima, d-gaps and
// medians, and the ParaPFD blocks, with the same bytes as the host build
// (codec.cpp), which restates the reference encoders (ParaPFor.cpp:31-113,
// ParaPFD_Compression/main.cpp:163-189, SegLRC_Generator.cu:190-331).
//
//   k_fit_segments   one thread per segment: the least-squares fit in double
//                    precision, summed in element order as the reference's
//                    host code does, every operation an explicitly rounded
//                    intrinsic so nothing is fused; then the window ranges L/R
//                    in single precision.
//   k_fit_lists      one thread per list: the same fit over the whole list
//                    (SegLRC's list-level regression).
//   k_block_plan     one warp per segment: the values to pack, the bit width
//                    (findBestB: smallest b whose exception count passes the
//                    FRAC test in single precision), exceptions, block size.
//   k_block_pack     one warp per segment: the block at its word offset; each
//                    lane assembles whole output words (LSB-first packing).
// Block offsets come from a scan of the block sizes in between.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <thread>
#include <string>
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
                            SegReg *__restrict__ lreg) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlists) return;
    const uint64_t o = list_off[l];
    const uint32_t n = (uint32_t)(list_off[l + 1] - o);
    if (n > kHostFit) return;
    const FitOut f = fit_seq(docs + o, n);
    lreg[l] = SegReg{f.a, f.b, f.L, f.R};
}

constexpr int kBuildWarps = 8;
constexpr uint32_t kErrBuildFormat = 1u;  // a block not representable (b = 32) or a residual spread > 31 bits
constexpr uint32_t kErrBuildOrder = 2u;   // a list is not strictly increasing

struct Plan {
    uint32_t lb, eb, hb, en;  // block parameters
    uint32_t words;           // block size
};

__global__ void __launch_bounds__(kBuildWarps * 32) k_block_plan(const uint32_t *__restrict__ docs, SegTab t,
                                                                 uint32_t nsegs, uint32_t codec, float frac,
                                                                 const SegReg *__restrict__ reg,
                                                                 uint32_t *__restrict__ vals,  // per element
                                                                 uint32_t *__restrict__ head, uint32_t *__restrict__ aux,
                                                                 Plan *__restrict__ plan, uint32_t *__restrict__ err) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t g = blockIdx.x * kBuildWarps + (threadIdx.x >> 5);
    if (g >= nsegs) return;
    const uint64_t lo = t.list_off[t.seg_list[g]];
    const uint32_t s0 = t.seg_start[g], n = t.seg_count[g];
    const uint32_t *y = docs + lo + s0;
    uint32_t *out = vals + lo + s0;
    uint32_t v[8];
    // strictly increasing lists only (as the host build requires)
    bool unordered = false;
    for (int q = 0; q < 8; ++q) {
        const uint32_t i = lane + 32u * q;
        unordered |= i < n && s0 + i > 0 && y[i] <= y[(int)i - 1];
    }
    if (__any_sync(0xffffffffu, unordered) && lane == 0) atomicOr(err, kErrBuildOrder);
    if (codec == EXCL_CODEC_PARAPFD) {
        // d-gaps across the whole list; element 0 of the list is its docID
        for (int q = 0; q < 8; ++q) {
            const uint32_t i = lane + 32u * q;
            v[q] = i < n ? (s0 + i == 0 ? y[i] : y[i] - y[(int)i - 1]) : 0u;
        }
        if (lane == 0) aux[g] = y[n / 2];
    } else {
        // residual against the segment fit, then minus the segment's minimum
        const SegReg r = reg[g];
        int32_t res[8];
        int32_t mn = 0x7fffffff;
        for (int q = 0; q < 8; ++q) {
            const uint32_t i = lane + 32u * q;
            if (i < n) {
                const int32_t p = __float2int_rz(__fmaf_rn(__uint2float_rn(i), r.a, r.b));
                res[q] = (int32_t)(y[i] - (uint32_t)p);
                mn = min(mn, res[q]);
            } else {
                res[q] = 0;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        bool bad = false;
        for (int q = 0; q < 8; ++q) {
            const int64_t d = (int64_t)res[q] - mn;
            bad |= (lane + 32u * q < n) && d > 0x7fffffffLL;
            v[q] = (uint32_t)d;
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(err, kErrBuildFormat);
        if (lane == 0) aux[g] = (uint32_t)mn;
    }
    if (lane == 0) head[g] = y[0];
    for (int q = 0; q < 8; ++q)
        if (lane + 32u * q < n) out[lane + 32u * q] = v[q];
    // findBestB (ParaPFor.cpp:31-53): for each width b, how many values need
    // more than b bits; the smallest b whose count passes the FRAC test
    const float lim = __fmul_rn(frac, __uint2float_rn(n));
    uint32_t nb[8];
    for (int q = 0; q < 8; ++q) nb[q] = lane + 32u * q < n ? nbits_d(v[q]) : 0u;
    uint32_t lb = 32;
    for (uint32_t b = 0; b < 32; ++b) {
        uint32_t above = 0;
        for (int q = 0; q < 8; ++q) above += __popc(__ballot_sync(0xffffffffu, nb[q] > b));
        if (__uint2float_rn(above) <= lim) {
            lb = b;
            break;
        }
    }
    Plan p{lb, 0u, 0u, 0u, 0u};
    if (lb >= 32) {
        if (lane == 0) atomicOr(err, kErrBuildFormat);
        p.lb = 0;
    } else {
        // exceptions in element order (q groups in order, lanes in order within a group)
        uint32_t en = 0, orh = 0, last = 0;
        for (int q = 0; q < 8; ++q) {
            const uint32_t i = lane + 32u * q;
            const bool ex = i < n && nb[q] > lb;
            const uint32_t m = __ballot_sync(0xffffffffu, ex);
            if (ex) orh |= v[q] >> lb;
            if (m) last = 32u * q + 31u - __clz(m);
            en += __popc(m);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) orh |= __shfl_xor_sync(0xffffffffu, orh, o);
        p.en = en;
        if (en) {
            p.eb = nbits_d(last);
            p.hb = nbits_d(orh);
            if (p.eb >= 32 || p.hb >= 32) {  // not representable in the descriptor (ParaPFor.cpp:79-88)
                if (lane == 0) atomicOr(err, kErrBuildFormat);
                p.en = p.eb = p.hb = 0;
            }
        }
    }
    p.words = 1u + (uint32_t)(((uint64_t)n * p.lb + 31u) >> 5);
    if (p.en) p.words += (uint32_t)(((uint64_t)p.en * p.eb + 31u) >> 5) + (uint32_t)(((uint64_t)p.en * p.hb + 31u) >> 5);
    if (lane == 0) plan[g] = p;
}

// Word k of an LSB-first packing of src[0..n) at `bits` bits per value.
__device__ __forceinline__ uint32_t packed_word(const uint32_t *src, uint32_t n, uint32_t bits, uint32_t k) {
    const uint64_t b0 = (uint64_t)k * 32u;
    const uint64_t last = (b0 + 31u) / bits + 1u;
    const uint32_t i0 = (uint32_t)(b0 / bits), i1 = (uint32_t)(last < n ? last : n);
    uint32_t w = 0;
    for (uint32_t i = i0; i < i1; ++i) {
        const int64_t sh = (int64_t)i * bits - (int64_t)b0;  // position of value i's bit 0 in this word
        const uint64_t val = src[i];
        if (sh >= 0) w |= (uint32_t)(val << sh);
        else w |= (uint32_t)(val >> (-sh));
    }
    return w;
}

__global__ void __launch_bounds__(kBuildWarps * 32) k_block_pack(const uint32_t *__restrict__ vals, SegTab t,
                                                                 uint32_t nsegs, const Plan *__restrict__ plan,
                                                                 const uint64_t *__restrict__ gword,
                                                                 uint32_t *__restrict__ words) {
    __shared__ uint32_t s_low[kBuildWarps][kTileKeys], s_pos[kBuildWarps][kTileKeys], s_high[kBuildWarps][kTileKeys];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t g = blockIdx.x * kBuildWarps + w;
    if (g >= nsegs) return;
    const Plan p = plan[g];
    const uint32_t n = t.seg_count[g];
    const uint32_t *v = vals + t.list_off[t.seg_list[g]] + t.seg_start[g];
    uint32_t *blk = words + gword[g];
    const uint32_t lim = p.lb < 32 ? (1u << p.lb) : 0u;
    uint32_t base = 0;
    for (int q = 0; q < 8; ++q) {
        const uint32_t i = lane + 32u * q;
        const uint32_t x = i < n ? v[i] : 0u;
        const bool ex = i < n && x >= lim;
        if (i < n) s_low[w][i] = x & (lim - 1u);
        const uint32_t m = __ballot_sync(0xffffffffu, ex);
        if (ex) {
            const uint32_t k = base + __popc(m & ((1u << lane) - 1u));
            s_pos[w][k] = i;
            s_high[w][k] = x >> p.lb;
        }
        base += __popc(m);
    }
    __syncwarp();
    const uint32_t wl = (uint32_t)(((uint64_t)n * p.lb + 31u) >> 5);
    if (lane == 0) blk[0] = p.en ? (p.lb << 26) + (p.eb << 21) + (p.hb << 16) + p.en : (p.lb << 26);
    if (p.lb)
        for (uint32_t k = lane; k < wl; k += 32) blk[1 + k] = packed_word(s_low[w], n, p.lb, k);
    if (p.en) {
        const uint32_t we = (uint32_t)(((uint64_t)p.en * p.eb + 31u) >> 5);
        const uint32_t wh = (uint32_t)(((uint64_t)p.en * p.hb + 31u) >> 5);
        if (p.eb)
            for (uint32_t k = lane; k < we; k += 32) blk[1 + wl + k] = packed_word(s_pos[w], p.en, p.eb, k);
        if (p.hb)
            for (uint32_t k = lane; k < wh; k += 32) blk[1 + wl + we + k] = packed_word(s_high[w], p.en, p.hb, k);
    }
}

__global__ void k_gather_last(const uint32_t *__restrict__ docs, const uint64_t *__restrict__ list_off, uint32_t nlists,
                              uint32_t *__restrict__ last) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < nlists) last[l] = docs[list_off[l + 1] - 1];
}

template <class T>
int dmalloc(T **p, size_t count) {
    return cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(count, 1) * sizeof(T)) == cudaSuccess ? 0 : 1;
}

}  // namespace
}  // namespace excl

using namespace excl;

extern "C" int excl_index_build_device(excl_ctx *ctx, const uint32_t *d_docs, const uint64_t *list_offsets,
                                       uint32_t nlists, const excl_build_params *p, excl_index **out) {
    if (!ctx || !d_docs || !list_offsets || !p || !out || nlists == 0) return EXCL_E_INVALID;
    *out = nullptr;
    if (p->codecs || (p->codec != EXCL_CODEC_PARAPFD && p->codec != EXCL_CODEC_SEGLRC)) return EXCL_E_INVALID;
    if (p->block < kMinBlock || p->block > kTileKeys || (p->block & (p->block - 1))) return EXCL_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const uint32_t B = p->block, codec = p->codec;
    // segment table (host): segments of every list in order
    std::vector<uint32_t> seg_list, seg_start, seg_count;
    std::vector<uint32_t> seg_base(nlists), nseg(nlists);
    for (uint32_t l = 0; l < nlists; ++l) {
        if (list_offsets[l + 1] <= list_offsets[l] || list_offsets[l + 1] - list_offsets[l] > 0xffffffffull)
            return EXCL_E_INVALID;
        const uint32_t n = (uint32_t)(list_offsets[l + 1] - list_offsets[l]);
        seg_base[l] = (uint32_t)seg_list.size();
        nseg[l] = (n + B - 1) / B;
        for (uint32_t s = 0; s < nseg[l]; ++s) {
            seg_list.push_back(l);
            seg_start.push_back(s * B);
            seg_count.push_back(std::min(B, n - s * B));
        }
    }
    const uint32_t ns = (uint32_t)seg_list.size();
    const uint64_t npost = list_offsets[nlists] - list_offsets[0];
    // device scratch for the build
    uint32_t *d_slist = nullptr, *d_sstart = nullptr, *d_scount = nullptr, *d_vals = nullptr, *d_head = nullptr,
             *d_aux = nullptr, *d_words = nullptr, *d_err = nullptr;
    uint64_t *d_loff = nullptr, *d_gword = nullptr;
    SegReg *d_reg = nullptr, *d_lreg = nullptr;
    Plan *d_plan = nullptr;
    int bad = 0;
    bad |= dmalloc(&d_slist, ns) | dmalloc(&d_sstart, ns) | dmalloc(&d_scount, ns) | dmalloc(&d_head, ns) |
           dmalloc(&d_aux, ns) | dmalloc(&d_reg, ns) | dmalloc(&d_plan, ns) | dmalloc(&d_gword, ns + 1) |
           dmalloc(&d_loff, (size_t)nlists + 1) | dmalloc(&d_lreg, nlists) | dmalloc(&d_vals, npost) |
           dmalloc(&d_err, 1);
    auto cleanup = [&]() {
        cudaFree(d_slist);
        cudaFree(d_sstart);
        cudaFree(d_scount);
        cudaFree(d_vals);
        cudaFree(d_head);
        cudaFree(d_aux);
        cudaFree(d_words);
        cudaFree(d_err);
        cudaFree(d_loff);
        cudaFree(d_gword);
        cudaFree(d_reg);
        cudaFree(d_lreg);
        cudaFree(d_plan);
    };
    if (bad) {
        cleanup();
        return EXCL_E_NOMEM;
    }
    // offsets relative to the first list, so d_docs may start anywhere
    std::vector<uint64_t> loff(nlists + 1);
    for (uint32_t l = 0; l <= nlists; ++l) loff[l] = list_offsets[l] - list_offsets[0];
    cudaError_t e = cudaMemcpyAsync(d_slist, seg_list.data(), (size_t)ns * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_sstart, seg_start.data(), (size_t)ns * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_scount, seg_count.data(), (size_t)ns * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_loff, loff.data(), loff.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, 4, st);
    const SegTab t{d_slist, d_sstart, d_scount, d_loff};
    const uint32_t *docs0 = d_docs + list_offsets[0];  // the kernels index from the first list
    // long lists: copied to the host (pinned) for their list-level fit, which
    // host threads run while the device kernels below proceed
    std::vector<uint32_t> host_fit;  // lists fitted on the host
    uint64_t host_words = 0;
    if (codec == EXCL_CODEC_SEGLRC)
        for (uint32_t l = 0; l < nlists; ++l)
            if (loff[l + 1] - loff[l] > kHostFit) {
                host_fit.push_back(l);
                host_words += loff[l + 1] - loff[l];
            }
    uint32_t *h_long = nullptr;
    cudaEvent_t long_ready = nullptr;
    std::vector<SegReg> host_reg(host_fit.size());
    std::thread fitter;
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
                        for (size_t i; (i = next.fetch_add(1)) < host_fit.size();)
                            host_reg[i] = fit_host(h_long + base[i], (uint32_t)(base[i + 1] - base[i]));
                    });
                for (auto &th : pool) th.join();
            });
    }
    if (e == cudaSuccess && codec == EXCL_CODEC_SEGLRC) {
        k_fit_segments<<<(ns + 127) / 128, 128, 0, st>>>(docs0, t, ns, d_reg);
        k_fit_lists<<<(nlists + 127) / 128, 128, 0, st>>>(docs0, d_loff, nlists, d_lreg);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_block_plan<<<(ns + kBuildWarps - 1) / kBuildWarps, kBuildWarps * 32, 0, st>>>(
            docs0, t, ns, codec, p->frac, d_reg, d_vals, d_head, d_aux, d_plan, d_err);
        e = cudaGetLastError();
    }
    // block offsets: a scan of the block sizes (host; 20 bytes per segment)
    std::vector<Plan> plan(ns);
    uint32_t flags = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(plan.data(), d_plan, (size_t)ns * sizeof(Plan), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flags, d_err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    auto join_fitter = [&]() {
        if (fitter.joinable()) fitter.join();
        if (long_ready) cudaEventDestroy(long_ready);
        long_ready = nullptr;
        if (h_long) cudaFreeHost(h_long);
        h_long = nullptr;
    };
    if (e != cudaSuccess || flags) {
        join_fitter();
        cleanup();
        if (e != cudaSuccess) return cuda_status(ctx, e, "device build");
        if (flags & kErrBuildOrder) {
            ctx_error(ctx, "posting lists are not strictly increasing");
            return EXCL_E_INVALID;
        }
        ctx_error(ctx, "a block is not representable in ParaPFD or a residual spread exceeds 31 bits");
        return EXCL_E_FORMAT;
    }
    std::vector<uint64_t> gword(ns + 1, 0);
    for (uint32_t g = 0; g < ns; ++g) gword[g + 1] = gword[g] + plan[g].words;
    if (dmalloc(&d_words, gword[ns] + kWordPad)) {
        join_fitter();
        cleanup();
        return EXCL_E_NOMEM;
    }
    e = cudaMemcpyAsync(d_gword, gword.data(), gword.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_words, 0, (gword[ns] + kWordPad) * 4, st);
    if (e == cudaSuccess) {
        k_block_pack<<<(ns + kBuildWarps - 1) / kBuildWarps, kBuildWarps * 32, 0, st>>>(d_vals, t, ns, d_plan,
                                                                                      d_gword, d_words);
        e = cudaGetLastError();
    }
    // the host image
    excl_index *ix = new (std::nothrow) excl_index();
    if (!ix) {
        join_fitter();
        cleanup();
        return EXCL_E_NOMEM;
    }
    ix->nlists = nlists;
    ix->lists.resize(nlists);
    ix->words.resize(gword[ns] + kWordPad);
    ix->seg_head.resize(ns);
    ix->seg_rec.resize(ns);
    ix->seg_reg.assign(ns, SegReg{1.0f, 0.0f, 0, 0});
    std::vector<uint32_t> aux(ns);
    std::vector<SegReg> lreg(nlists);
    std::vector<uint32_t> last(nlists);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ix->words.data(), d_words, ix->words.size() * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ix->seg_head.data(), d_head, (size_t)ns * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(aux.data(), d_aux, (size_t)ns * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && codec == EXCL_CODEC_SEGLRC) {
        e = cudaMemcpyAsync(ix->seg_reg.data(), d_reg, (size_t)ns * sizeof(SegReg), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(lreg.data(), d_lreg, (size_t)nlists * sizeof(SegReg), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) {
        // the lists' last docIDs
        uint32_t *d_last = nullptr;
        if (dmalloc(&d_last, nlists)) e = cudaErrorMemoryAllocation;
        if (e == cudaSuccess) {
            k_gather_last<<<(nlists + 255) / 256, 256, 0, st>>>(docs0, d_loff, nlists, d_last);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(last.data(), d_last, (size_t)nlists * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(d_last);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    join_fitter();
    cleanup();
    if (e != cudaSuccess) {
        delete ix;
        return cuda_status(ctx, e, "device build");
    }
    for (size_t i = 0; i < host_fit.size(); ++i) lreg[host_fit[i]] = host_reg[i];
    std::vector<uint32_t> ldir;
    ix->postings = npost;
    for (uint32_t l = 0; l < nlists; ++l) {
        ListDesc &d = ix->lists[l];
        d.n = (uint32_t)(loff[l + 1] - loff[l]);
        d.codec = codec;
        d.log2_block = (uint32_t)__builtin_ctz(B);
        d.seg_base = seg_base[l];
        d.nseg = nseg[l];
        d.word_base = gword[seg_base[l]];
        d.first_doc = ix->seg_head[seg_base[l]];
        d.last_doc = last[l];
        d.model = kNoModel;
        if (codec == EXCL_CODEC_SEGLRC) std::memcpy(d.reg, &lreg[l], sizeof(SegReg));
        for (uint32_t s = 0; s < nseg[l]; ++s) {
            const uint32_t g = seg_base[l] + s;
            SegRec &r = ix->seg_rec[g];
            r.start = seg_start[g];
            r.off = (uint32_t)(gword[g] - d.word_base);
            r.aux = aux[g];
            r.count = seg_count[g];
        }
        fixed_list_directory(d, ix->seg_head.data() + d.seg_base, d.nseg, ldir);
        d.dir_base = (uint32_t)ix->dir.size();
        ix->dir.insert(ix->dir.end(), ldir.begin(), ldir.end());
        d.tile_base = 0;
        d.ntiles = d.nseg;
    }
    *out = ix;
    return EXCL_OK;
}
