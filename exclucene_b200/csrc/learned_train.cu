// Learned position models: training and leaf fitting on the device.
//
// Per list (fixed-block codecs, n >= min_postings) a two-stage model maps a
// docID to its rank:
//   root  FP32 MLP 1 -> 32 -> 32 -> 1 (ReLU) on x = (key - first) / (last - first),
//         trained by these kernels on the list's own (docID, rank) pairs with an
//         MSE loss on rank / (n - 1); weights are kept non-negative after every
//         step, so the network (like the CDF it fits) is non-decreasing in x;
//   leaf  out * L routes the key to one of L linear fits rank ~ a*x + b,
//         solved from per-leaf sums over all keys;
//   error per leaf, the min and max of rank - floor(a*x + b) over the leaf's
//         keys, computed with the same inference code the probe phase runs,
//         so a present key's rank always lies in [pred + elo, pred + ehi].
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "excl_device.cuh"
#include "kernels.h"
#include "runtime.h"

namespace excl {

struct ModelSet {
    std::vector<float> root;
    std::vector<ModelHdr> hdr;
    std::vector<Leaf> leaves;
    std::vector<uint16_t> grid;
    std::vector<uint32_t> bnd;
    float *d_root = nullptr;
    ModelHdr *d_hdr = nullptr;
    Leaf *d_leaves = nullptr;
    uint16_t *d_grid = nullptr;
    uint32_t *d_bnd = nullptr;
    int device = 0;
};

namespace {

constexpr int H = kHidden;
constexpr int kP = kRootParams;  // 1153
// parameter layout (same as model_root): w1[32] b1[32] w2[32][32] b2[32] w3[32] b3
constexpr int oW1 = 0, oB1 = 32, oW2 = 64, oB2 = 64 + 1024, oW3 = 64 + 1024 + 32, oB3 = 64 + 1024 + 64;
constexpr int kTrainThreads = 128;
constexpr int kPad = H + 1;

__device__ __forceinline__ uint32_t hash32(uint32_t a, uint32_t b) {
    uint32_t h = a * 0x9e3779b1u ^ (b + 0x7f4a7c15u + (a << 6) + (a >> 2));
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// One block: kTrainThreads samples; per-sample forward/backward; per-block
// gradient sums written to partial[blockIdx][kP]. When keys == nullptr the
// samples come from (xs, ys) directly (the gradient-check entry point).
__global__ void __launch_bounds__(kTrainThreads) k_mlp_grad(const float *__restrict__ P, const uint32_t *__restrict__ keys,
                                                            uint32_t n, float kmin, float kscale, uint32_t step,
                                                            uint32_t seed, const float *__restrict__ xs,
                                                            const float *__restrict__ ys, uint32_t nsamples,
                                                            float *__restrict__ partial, float *__restrict__ loss_out) {
    extern __shared__ float sh[];
    float *sW = sh;                              // kP
    float *sH1 = sW + 1156;                      // [T][kPad]
    float *sDz2 = sH1 + kTrainThreads * kPad;    // [T][kPad]
    float *sDz1 = sDz2 + kTrainThreads * kPad;   // [T][kPad]
    float *sH2 = sDz1 + kTrainThreads * kPad;    // [T][kPad]
    float *sX = sH2 + kTrainThreads * kPad;      // [T]
    float *sDo = sX + kTrainThreads;             // [T]
    for (int i = threadIdx.x; i < kP; i += blockDim.x) sW[i] = P[i];
    __syncthreads();
    const uint32_t sidx = blockIdx.x * kTrainThreads + threadIdx.x;
    const bool valid = sidx < nsamples;
    float x = 0.0f, y = 0.0f;
    if (valid) {
        if (keys) {
            const uint32_t p = hash32(seed + step * 0x632be5abu, sidx) % n;
            x = __fmul_rn(__fsub_rn(__uint2float_rn(keys[p]), kmin), kscale);
            y = n > 1 ? (float)p / (float)(n - 1) : 0.0f;
        } else {
            x = xs[sidx];
            y = ys[sidx];
        }
    }
    const float *w1 = sW + oW1, *b1 = sW + oB1, *w2 = sW + oW2, *b2 = sW + oB2, *w3 = sW + oW3;
    float h1[H], z1[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
        z1[i] = __fmaf_rn(w1[i], x, b1[i]);
        h1[i] = fmaxf(z1[i], 0.0f);
    }
    float z2[H];
    float out = sW[oB3];
#pragma unroll 4
    for (int o = 0; o < H; ++o) {
        float acc = b2[o];
#pragma unroll
        for (int i = 0; i < H; ++i) acc = __fmaf_rn(w2[o * H + i], h1[i], acc);
        z2[o] = acc;
        out = __fmaf_rn(w3[o], fmaxf(acc, 0.0f), out);
    }
    const float diff = valid ? out - y : 0.0f;
    const float dout = valid ? 2.0f * diff / (float)nsamples : 0.0f;
    float *myH1 = sH1 + threadIdx.x * kPad, *myDz2 = sDz2 + threadIdx.x * kPad, *myDz1 = sDz1 + threadIdx.x * kPad,
          *myH2 = sH2 + threadIdx.x * kPad;
#pragma unroll
    for (int o = 0; o < H; ++o) {
        const float h2 = fmaxf(z2[o], 0.0f);
        myH2[o] = h2;
        myDz2[o] = z2[o] > 0.0f ? dout * w3[o] : 0.0f;
        myH1[o] = h1[o];
    }
    // dh1 = W2^T dz2
#pragma unroll 4
    for (int i = 0; i < H; ++i) {
        float acc = 0.0f;
#pragma unroll
        for (int o = 0; o < H; ++o) acc = __fmaf_rn(w2[o * H + i], myDz2[o], acc);
        myDz1[i] = z1[i] > 0.0f ? acc : 0.0f;
    }
    sX[threadIdx.x] = x;
    sDo[threadIdx.x] = dout;
    // loss (sum of squared differences) for reporting
    float l2 = diff * diff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l2 += __shfl_xor_sync(0xffffffffu, l2, o);
    if ((threadIdx.x & 31) == 0 && loss_out) atomicAdd(loss_out, l2);
    __syncthreads();
    // reduce over the block's samples: parameter j summed in a fixed order
    float *dst = partial + (size_t)blockIdx.x * kP;
    for (int j = threadIdx.x; j < kP; j += blockDim.x) {
        float g = 0.0f;
        if (j < oB1) {
            const int i = j - oW1;
            for (int s = 0; s < kTrainThreads; ++s) g = __fmaf_rn(sDz1[s * kPad + i], sX[s], g);
        } else if (j < oW2) {
            const int i = j - oB1;
            for (int s = 0; s < kTrainThreads; ++s) g = __fadd_rn(g, sDz1[s * kPad + i]);
        } else if (j < oB2) {
            const int o = (j - oW2) / H, i = (j - oW2) % H;
            for (int s = 0; s < kTrainThreads; ++s) g = __fmaf_rn(sDz2[s * kPad + o], sH1[s * kPad + i], g);
        } else if (j < oW3) {
            const int o = j - oB2;
            for (int s = 0; s < kTrainThreads; ++s) g = __fadd_rn(g, sDz2[s * kPad + o]);
        } else if (j < oB3) {
            const int o = j - oW3;
            for (int s = 0; s < kTrainThreads; ++s) g = __fmaf_rn(sDo[s], sH2[s * kPad + o], g);
        } else {
            for (int s = 0; s < kTrainThreads; ++s) g = __fadd_rn(g, sDo[s]);
        }
        dst[j] = g;
    }
}

constexpr size_t kGradSmem =
    (1156 + 4 * (size_t)kTrainThreads * kPad + 2 * (size_t)kTrainThreads) * sizeof(float);

// Sum the per-block partials (fixed order) into grad; optionally an Adam step
// with non-negative projection of the weights.
__global__ void k_mlp_update(float *__restrict__ P, float *__restrict__ m, float *__restrict__ v,
                             const float *__restrict__ partial, uint32_t nblocks, float *__restrict__ grad_out,
                             float lr, float b1c, float b2c, int do_update) {
    for (int j = threadIdx.x; j < kP; j += blockDim.x) {
        float g = 0.0f;
        for (uint32_t b = 0; b < nblocks; ++b) g = __fadd_rn(g, partial[(size_t)b * kP + j]);
        if (grad_out) grad_out[j] = g;
        if (!do_update) continue;
        const float mj = 0.9f * m[j] + 0.1f * g;
        const float vj = 0.999f * v[j] + 0.001f * g * g;
        m[j] = mj;
        v[j] = vj;
        float p = P[j] - lr * (mj / b1c) / (sqrtf(vj / b2c) + 1e-8f);
        const bool weight = j < oB1 || (j >= oW2 && j < oB2) || (j >= oW3 && j < oB3);
        if (weight && p < 0.0f) p = 0.0f;
        P[j] = p;
    }
}

// Per-leaf sums over all keys (run-length aggregated double atomics).
__global__ void k_leaf_sums(const uint16_t *__restrict__ grid, const uint32_t *__restrict__ bnd, ModelHdr m,
                            const uint32_t *__restrict__ keys, uint32_t n, uint32_t run,
                            double *__restrict__ sums /* L x 5 */) {
    const float kmin = m.kmin, kscale = m.kscale;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t p0 = t * run;
    if (p0 >= n) return;
    const uint64_t p1 = std::min<uint64_t>(n, p0 + run);
    uint32_t cur = 0xffffffffu;
    double c = 0, sx = 0, sy = 0, sxx = 0, sxy = 0;
    for (uint64_t p = p0; p < p1; ++p) {
        const float x = __fmul_rn(__fsub_rn(__uint2float_rn(keys[p]), kmin), kscale);
        const uint32_t leaf = model_route(grid, bnd, m, keys[p]);
        if (leaf != cur) {
            if (cur != 0xffffffffu) {
                double *s = sums + (size_t)cur * 5;
                atomicAdd(s + 0, c);
                atomicAdd(s + 1, sx);
                atomicAdd(s + 2, sy);
                atomicAdd(s + 3, sxx);
                atomicAdd(s + 4, sxy);
            }
            cur = leaf;
            c = sx = sy = sxx = sxy = 0;
        }
        const double dx = x, dy = (double)p;
        c += 1;
        sx += dx;
        sy += dy;
        sxx += dx * dx;
        sxy += dx * dy;
    }
    double *s = sums + (size_t)cur * 5;
    atomicAdd(s + 0, c);
    atomicAdd(s + 1, sx);
    atomicAdd(s + 2, sy);
    atomicAdd(s + 3, sxx);
    atomicAdd(s + 4, sxy);
}

__global__ void k_leaf_solve(const double *__restrict__ sums, uint32_t L, Leaf *__restrict__ leaves) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= L) return;
    const double *s = sums + (size_t)l * 5;
    const double c = s[0];
    Leaf lf;
    lf.a = 0.0f;
    lf.b = 0.0f;
    lf.elo = 0x7fffffff;
    lf.ehi = (int32_t)0x80000000;
    if (c > 0) {
        const double mx = s[1] / c, my = s[2] / c;
        const double vxx = s[3] / c - mx * mx, vxy = s[4] / c - mx * my;
        double a = (c > 1 && vxx > 1e-30) ? vxy / vxx : 0.0;
        double b = my - a * mx;
        if (!std::isfinite(a) || !std::isfinite(b)) {
            a = 0.0;
            b = my;
        }
        lf.a = (float)a;
        lf.b = (float)b;
    }
    leaves[l] = lf;
}

// Exact per-leaf error window with the query-time arithmetic.
__global__ void k_leaf_err(const uint16_t *__restrict__ grid, const uint32_t *__restrict__ bnd, ModelHdr m,
                           const uint32_t *__restrict__ keys, uint32_t n, uint32_t run, Leaf *__restrict__ leaves) {
    const float kmin = m.kmin, kscale = m.kscale;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t p0 = t * run;
    if (p0 >= n) return;
    const uint64_t p1 = std::min<uint64_t>(n, p0 + run);
    uint32_t cur = 0xffffffffu;
    int32_t lo = 0, hi = 0;
    for (uint64_t p = p0; p < p1; ++p) {
        const float x = __fmul_rn(__fsub_rn(__uint2float_rn(keys[p]), kmin), kscale);
        const uint32_t leaf = model_route(grid, bnd, m, keys[p]);
        if (leaf != cur) {
            if (cur != 0xffffffffu) {
                atomicMin(&leaves[cur].elo, lo);
                atomicMax(&leaves[cur].ehi, hi);
            }
            cur = leaf;
            lo = 0x7fffffff;
            hi = (int32_t)0x80000000;
        }
        Leaf lf;  // only the fit is read here; elo/ehi are being reduced concurrently
        lf.a = leaves[leaf].a;
        lf.b = leaves[leaf].b;
        const int64_t e = (int64_t)p - (int64_t)model_pred_rank(lf, x);
        const int32_t ec = (int32_t)std::max<int64_t>(-0x7fffffffLL, std::min<int64_t>(0x7fffffffLL, e));
        lo = min(lo, ec);
        hi = max(hi, ec);
    }
    atomicMin(&leaves[cur].elo, lo);
    atomicMax(&leaves[cur].ehi, hi);
}

// Routing of the root MLP at key k (the network evaluated as the probe would).
__device__ __forceinline__ uint32_t mlp_leaf(const float *W, float kmin, float kscale, uint32_t L, uint32_t k) {
    return model_leaf_of(model_root(W, __fmul_rn(__fsub_rn(__uint2float_rn(k), kmin), kscale)), L);
}

// bnd[l] = smallest key in [first, last] whose leaf is >= l (0xffffffff if none);
// a binary search over the key range, valid because the routing is non-decreasing.
__global__ void k_model_bnd(const float *__restrict__ W, uint32_t first, uint32_t last, float kmin, float kscale,
                            uint32_t L, uint32_t *__restrict__ bnd) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= L) return;
    uint64_t lo = first, hi = (uint64_t)last + 1;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (mlp_leaf(W, kmin, kscale, L, (uint32_t)mid) >= l) hi = mid;
        else lo = mid + 1;
    }
    bnd[l] = lo > last ? 0xffffffffu : (uint32_t)lo;
}

// grid[j] = leaf of the key first + (j << shift) (clamped to last), j in [0, grid_n].
__global__ void k_model_grid(const float *__restrict__ W, uint32_t first, uint32_t last, uint32_t shift,
                             uint32_t grid_n, float kmin, float kscale, uint32_t L, uint16_t *__restrict__ grid) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > grid_n) return;
    const uint64_t k = std::min<uint64_t>((uint64_t)first + ((uint64_t)j << shift), last);
    grid[j] = (uint16_t)mlp_leaf(W, kmin, kscale, L, (uint32_t)k);
}

void init_root(float *P, uint32_t seed) {
    // a non-decreasing ramp basis: layer-1 hinges spread over [0, 1], small
    // positive mixing weights; deterministic in the seed
    uint32_t s = seed * 2654435761u + 1;
    auto rnd = [&]() {
        s ^= s << 13;
        s ^= s >> 17;
        s ^= s << 5;
        return (s & 0xffffff) / 16777216.0f;
    };
    for (int i = 0; i < H; ++i) {
        P[oW1 + i] = 1.0f + rnd();
        P[oB1 + i] = -(float)i / H * P[oW1 + i];
    }
    for (int i = 0; i < H * H; ++i) P[oW2 + i] = 0.05f * rnd();
    for (int i = 0; i < H; ++i) P[oB2 + i] = 0.0f;
    for (int i = 0; i < H; ++i) P[oW3 + i] = 0.05f * rnd();
    P[oB3] = 0.0f;
}

}  // namespace

ModelView model_view(const ModelSet *m) {
    ModelView v{};
    if (m) {
        v.root = m->d_root;
        v.hdr = m->d_hdr;
        v.leaves = m->d_leaves;
        v.grid = m->d_grid;
        v.bnd = m->d_bnd;
    }
    return v;
}

static void models_release_device(ModelSet *m) {
    cudaFree(m->d_root);
    cudaFree(m->d_hdr);
    cudaFree(m->d_leaves);
    cudaFree(m->d_grid);
    cudaFree(m->d_bnd);
    m->d_root = nullptr;
    m->d_hdr = nullptr;
    m->d_leaves = nullptr;
    m->d_grid = nullptr;
    m->d_bnd = nullptr;
}

void models_free(ModelSet *m) {
    if (!m) return;
    models_release_device(m);
    delete m;
}

int models_upload(excl_ctx *ctx, excl_index *ix) {
    ModelSet *m = ix->models;
    if (!m) return EXCL_OK;
    models_release_device(m);
    int st = EXCL_OK;
    auto put = [&](void **dst, const void *src, size_t bytes, const char *what) {
        if (st || bytes == 0) return;
        st = cuda_status(ctx, cudaMalloc(dst, bytes), what);
        if (!st) st = cuda_status(ctx, cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice), what);
    };
    put((void **)&m->d_root, m->root.data(), m->root.size() * 4, "model root");
    put((void **)&m->d_hdr, m->hdr.data(), m->hdr.size() * sizeof(ModelHdr), "model header");
    put((void **)&m->d_leaves, m->leaves.data(), m->leaves.size() * sizeof(Leaf), "model leaves");
    put((void **)&m->d_grid, m->grid.data(), m->grid.size() * 2, "model grid");
    put((void **)&m->d_bnd, m->bnd.data(), m->bnd.size() * 4, "model boundaries");
    // the list descriptors carry the model slots
    if (!st && ix->dev)
        st = cuda_status(ctx, cudaMemcpy(ix->dev->lists, ix->lists.data(), ix->lists.size() * sizeof(ListDesc),
                                         cudaMemcpyHostToDevice),
                         "lists");
    m->device = ctx->device;
    return st;
}

struct TrainBufs {
    float *P = nullptr, *m = nullptr, *v = nullptr, *partial = nullptr, *loss = nullptr;
    double *sums = nullptr;
    Leaf *leaves = nullptr;
    uint16_t *grid = nullptr;
    uint32_t *bnd = nullptr;
    uint32_t max_blocks = 512;
};

struct TrainedModel {
    std::vector<float> root;
    std::vector<Leaf> leaves;
    std::vector<uint16_t> grid;
    std::vector<uint32_t> bnd;
    ModelHdr hdr{};
    float loss = 0;
    double train_ms = 0, fit_ms = 0;
};

static uint32_t pow2_at_least(uint64_t v) {
    uint32_t p = 1;
    while (p < v && p < (1u << 30)) p <<= 1;
    return p;
}

// Trains one list's model on the device: root MLP, routing tables, leaf fits
// and exact error windows (the last two through the same table routing the
// probe uses).
static int train_one(excl_ctx *ctx, const uint32_t *d_keys, uint32_t n, uint32_t first, uint32_t last, uint32_t L,
                     const excl_learn_params &p, uint32_t seed, TrainBufs &tb, TrainedModel &out) {
    cudaStream_t st = ctx->stream;
    const float kmin = (float)first;
    const float span = (float)last - (float)first;
    const float kscale = span > 0.0f ? 1.0f / span : 0.0f;
    std::vector<float> P(kRootStride, 0.0f);
    init_root(P.data(), seed);
    cudaMemcpyAsync(tb.P, P.data(), kP * 4, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(tb.m, 0, kP * 4, st);
    cudaMemsetAsync(tb.v, 0, kP * 4, st);
    const uint32_t batch = std::min<uint32_t>(p.batch, tb.max_blocks * kTrainThreads);
    const uint32_t nb = (batch + kTrainThreads - 1) / kTrainThreads;
    auto t0 = std::chrono::steady_clock::now();
    float b1c = 1.0f, b2c = 1.0f;
    for (uint32_t s = 0; s < p.steps; ++s) {
        const float frac = (float)s / (float)std::max(1u, p.steps);
        const float lr = p.lr * (0.5f * (1.0f + cosf(3.14159265f * frac)) * 0.95f + 0.05f);
        b1c *= 0.9f;
        b2c *= 0.999f;
        if (s + 1 == p.steps) cudaMemsetAsync(tb.loss, 0, 4, st);
        k_mlp_grad<<<nb, kTrainThreads, kGradSmem, st>>>(tb.P, d_keys, n, kmin, kscale, s, seed, nullptr, nullptr,
                                                          batch, tb.partial, s + 1 == p.steps ? tb.loss : nullptr);
        k_mlp_update<<<1, 1024, 0, st>>>(tb.P, tb.m, tb.v, tb.partial, nb, nullptr, lr, 1.0f - b1c, 1.0f - b2c, 1);
    }
    int e = cuda_status(ctx, cudaStreamSynchronize(st), "train");
    if (e) return e;
    auto t1 = std::chrono::steady_clock::now();
    cudaMemcpy(&out.loss, tb.loss, 4, cudaMemcpyDeviceToHost);
    out.loss /= (float)batch;
    // routing tables
    ModelHdr &h = out.hdr;
    h.kmin = kmin;
    h.kscale = kscale;
    h.nleaves = L;
    h.n = n;
    h.max_window = p.max_window;
    h.first = first;
    h.grid_n = std::max<uint32_t>(64, pow2_at_least(2ull * L));
    uint32_t sb = 0;
    while (sb < 32 && (((uint64_t)(last - first)) >> sb) >= h.grid_n) ++sb;
    h.grid_shift = sb;
    h.grid_base = 0;
    h.bnd_base = 0;
    k_model_bnd<<<(L + 127) / 128, 128, 0, st>>>(tb.P, first, last, kmin, kscale, L, tb.bnd);
    k_model_grid<<<(h.grid_n + 1 + 127) / 128, 128, 0, st>>>(tb.P, first, last, h.grid_shift, h.grid_n, kmin, kscale,
                                                             L, tb.grid);
    // leaves
    const uint32_t run = 64;
    const uint64_t threads = (n + run - 1) / run;
    const uint32_t blocks = (uint32_t)((threads + 255) / 256);
    cudaMemsetAsync(tb.sums, 0, (size_t)L * 5 * sizeof(double), st);
    k_leaf_sums<<<blocks, 256, 0, st>>>(tb.grid, tb.bnd, h, d_keys, n, run, tb.sums);
    k_leaf_solve<<<(L + 255) / 256, 256, 0, st>>>(tb.sums, L, tb.leaves);
    k_leaf_err<<<blocks, 256, 0, st>>>(tb.grid, tb.bnd, h, d_keys, n, run, tb.leaves);
    e = cuda_status(ctx, cudaStreamSynchronize(st), "leaf fit");
    if (e) return e;
    auto t2 = std::chrono::steady_clock::now();
    out.root.resize(kRootStride);
    cudaMemcpy(out.root.data(), tb.P, kRootStride * 4, cudaMemcpyDeviceToHost);
    out.leaves.resize(L);
    cudaMemcpy(out.leaves.data(), tb.leaves, (size_t)L * sizeof(Leaf), cudaMemcpyDeviceToHost);
    out.grid.resize(h.grid_n + 1);
    cudaMemcpy(out.grid.data(), tb.grid, (h.grid_n + 1) * 2, cudaMemcpyDeviceToHost);
    out.bnd.resize(L);
    cudaMemcpy(out.bnd.data(), tb.bnd, (size_t)L * 4, cudaMemcpyDeviceToHost);
    for (Leaf &lf : out.leaves)
        if (lf.elo > lf.ehi) {  // no key routes here: an empty window
            lf.elo = 1;
            lf.ehi = 0;
        }
    out.train_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    out.fit_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    return EXCL_OK;
}

}  // namespace excl

using namespace excl;

extern "C" int excl_learn_models(excl_ctx *ctx, excl_index *ix, const excl_learn_params *params,
                                 excl_learn_report *rep) {
    if (!ctx || !ix || !params) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    if (!ix->dev) {
        ctx_error(ctx, "index not uploaded");
        return EXCL_E_INVALID;
    }
    excl_learn_params p = *params;
    if (p.nleaves == 0) p.nleaves = 4096;
    if (p.nleaves > 65536) p.nleaves = 65536;
    if (p.steps == 0) p.steps = 300;
    if (p.batch == 0) p.batch = 16384;
    if (p.lr <= 0) p.lr = 3e-3f;
    if (p.max_window == 0) p.max_window = 4096;
    if (p.min_postings == 0) p.min_postings = 1u << 20;
    cudaSetDevice(ctx->device);
    std::vector<uint32_t> which;
    uint64_t maxn = 0;
    for (uint32_t l = 0; l < ix->nlists; ++l) {
        const ListDesc &d = ix->lists[l];
        if (d.n >= p.min_postings && d.log2_block != 0 && d.n >= 2 && d.last_doc != 0xffffffffu) {
            which.push_back(l);
            maxn = std::max<uint64_t>(maxn, d.n);
        }
    }
    ModelSet *ms = ix->models ? ix->models : new ModelSet();
    ms->root.clear();
    ms->hdr.clear();
    ms->leaves.clear();
    ms->grid.clear();
    ms->bnd.clear();
    for (auto &d : ix->lists) d.model = kNoModel;
    excl_learn_report r{};
    int st = EXCL_OK;
    uint32_t *d_keys = nullptr;
    TrainBufs tb;
    const uint32_t Lmax = p.nleaves;
    if (!which.empty()) {
        st |= cuda_status(ctx, cudaMalloc((void **)&d_keys, maxn * 4), "model keys");
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.P, kRootStride * 4), "model");
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.m, kRootStride * 4), "model");
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.v, kRootStride * 4), "model");
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.partial, (size_t)tb.max_blocks * kP * 4), "model");
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.loss, 4), "model");
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.sums, (size_t)Lmax * 5 * 8), "model");
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.leaves, (size_t)Lmax * sizeof(Leaf)), "model");
        // grid_n = max(64, next power of two >= 2L) <= 4 * Lmax, plus one entry
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.grid, ((size_t)4 * Lmax + 64 + 2) * 2), "model");
        st |= cuda_status(ctx, cudaMalloc((void **)&tb.bnd, (size_t)Lmax * 4), "model");
        cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem);
    }
    double win_sum = 0, wide = 0;
    uint64_t leaves_total = 0;
    for (size_t k = 0; k < which.size() && !st; ++k) {
        const uint32_t l = which[k];
        const ListDesc &d = ix->lists[l];
        // about 32 postings per leaf, at most nleaves
        const uint32_t L = std::max<uint32_t>(64, std::min<uint32_t>(Lmax, pow2_at_least((d.n + 31) / 32)));
        st = excl_decode_lists_device(ctx, ix, l, l + 1, d_keys);
        if (st) break;
        TrainedModel tm;
        st = train_one(ctx, d_keys, d.n, d.first_doc, d.last_doc, L, p, p.seed + l, tb, tm);
        if (st) break;
        tm.hdr.leaf_base = (uint32_t)ms->leaves.size();
        tm.hdr.grid_base = (uint32_t)ms->grid.size();
        tm.hdr.bnd_base = (uint32_t)ms->bnd.size();
        ix->lists[l].model = (uint32_t)ms->hdr.size();
        ms->hdr.push_back(tm.hdr);
        ms->root.insert(ms->root.end(), tm.root.begin(), tm.root.end());
        ms->grid.insert(ms->grid.end(), tm.grid.begin(), tm.grid.end());
        ms->bnd.insert(ms->bnd.end(), tm.bnd.begin(), tm.bnd.end());
        for (const Leaf &lf : tm.leaves) {
            if (lf.ehi >= lf.elo) {
                const double wdt = (double)lf.ehi - (double)lf.elo + 1;
                win_sum += wdt;
                ++leaves_total;
                if (wdt > p.max_window) wide += 1;
            }
        }
        ms->leaves.insert(ms->leaves.end(), tm.leaves.begin(), tm.leaves.end());
        r.train_ms += tm.train_ms;
        r.fit_ms += tm.fit_ms;
        r.final_loss = std::max(r.final_loss, tm.loss);
    }
    cudaFree(d_keys);
    cudaFree(tb.P);
    cudaFree(tb.m);
    cudaFree(tb.v);
    cudaFree(tb.partial);
    cudaFree(tb.loss);
    cudaFree(tb.sums);
    cudaFree(tb.leaves);
    cudaFree(tb.grid);
    cudaFree(tb.bnd);
    if (st) {
        for (auto &d : ix->lists) d.model = kNoModel;
        if (!ix->models) delete ms;
        return st;
    }
    ix->models = ms;
    st = models_upload(ctx, ix);
    r.models = (uint32_t)which.size();
    r.mean_window = leaves_total ? win_sum / (double)leaves_total : 0;
    r.wide_leaf_frac = leaves_total ? wide / (double)leaves_total : 0;
    r.params_bytes = ms->root.size() * 4 + ms->hdr.size() * sizeof(ModelHdr) + ms->leaves.size() * sizeof(Leaf) +
                     ms->grid.size() * 2 + ms->bnd.size() * 4;
    if (rep) *rep = r;
    return st;
}

extern "C" int excl_model_tables(const excl_index *ix, uint32_t list, uint16_t *grid, uint32_t *bnd,
                                 uint32_t meta[4]) {
    if (!ix || list >= ix->nlists || !meta) return EXCL_E_INVALID;
    const uint32_t slot = ix->lists[list].model;
    if (slot == kNoModel || !ix->models) return EXCL_E_INVALID;
    const ModelSet *m = ix->models;
    const ModelHdr &h = m->hdr[slot];
    meta[0] = h.first;
    meta[1] = h.grid_shift;
    meta[2] = h.grid_n;
    meta[3] = h.nleaves;
    if (grid) std::memcpy(grid, m->grid.data() + h.grid_base, (h.grid_n + 1) * 2);
    if (bnd) std::memcpy(bnd, m->bnd.data() + h.bnd_base, (size_t)h.nleaves * 4);
    return EXCL_OK;
}

extern "C" int excl_model_export(const excl_index *ix, uint32_t list, float *root, float *hdr4, int32_t *leaves,
                                 uint32_t *nleaves) {
    if (!ix || list >= ix->nlists) return EXCL_E_INVALID;
    const uint32_t slot = ix->lists[list].model;
    if (slot == kNoModel || !ix->models) return EXCL_E_INVALID;
    const ModelSet *m = ix->models;
    const ModelHdr &h = m->hdr[slot];
    if (nleaves) *nleaves = h.nleaves;
    if (root) std::memcpy(root, m->root.data() + (size_t)slot * kRootStride, kRootParams * 4);
    if (hdr4) {
        hdr4[0] = h.kmin;
        hdr4[1] = h.kscale;
        hdr4[2] = (float)h.nleaves;
        hdr4[3] = (float)h.max_window;
    }
    if (leaves) std::memcpy(leaves, m->leaves.data() + h.leaf_base, (size_t)h.nleaves * sizeof(Leaf));
    return EXCL_OK;
}

extern "C" int excl_model_grad(excl_ctx *ctx, const float *params, const float *x, const float *y, uint32_t n,
                               float *grad, float *loss) {
    if (!ctx || !params || !x || !y || !grad || n == 0) return EXCL_E_INVALID;
    std::lock_guard<std::recursive_mutex> g(ctx->op_mu);
    cudaSetDevice(ctx->device);
    const uint32_t nb = (n + kTrainThreads - 1) / kTrainThreads;
    float *d_P = nullptr, *d_x = nullptr, *d_y = nullptr, *d_part = nullptr, *d_g = nullptr, *d_loss = nullptr;
    int st = 0;
    st |= cuda_status(ctx, cudaMalloc((void **)&d_P, kRootStride * 4), "grad");
    st |= cuda_status(ctx, cudaMalloc((void **)&d_x, (size_t)n * 4), "grad");
    st |= cuda_status(ctx, cudaMalloc((void **)&d_y, (size_t)n * 4), "grad");
    st |= cuda_status(ctx, cudaMalloc((void **)&d_part, (size_t)nb * kP * 4), "grad");
    st |= cuda_status(ctx, cudaMalloc((void **)&d_g, kRootStride * 4), "grad");
    st |= cuda_status(ctx, cudaMalloc((void **)&d_loss, 4), "grad");
    if (!st) {
        cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem);
        cudaMemcpy(d_P, params, kP * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(d_x, x, (size_t)n * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(d_y, y, (size_t)n * 4, cudaMemcpyHostToDevice);
        cudaMemset(d_loss, 0, 4);
        k_mlp_grad<<<nb, kTrainThreads, kGradSmem, ctx->stream>>>(d_P, nullptr, 0, 0.0f, 0.0f, 0, 0, d_x, d_y, n,
                                                                   d_part, d_loss);
        k_mlp_update<<<1, 1024, 0, ctx->stream>>>(d_P, nullptr, nullptr, d_part, nb, d_g, 0.0f, 1.0f, 1.0f, 0);
        st = cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "grad");
        if (!st) {
            cudaMemcpy(grad, d_g, kP * 4, cudaMemcpyDeviceToHost);
            float l = 0;
            cudaMemcpy(&l, d_loss, 4, cudaMemcpyDeviceToHost);
            if (loss) *loss = l / (float)n;
        }
    }
    cudaFree(d_P);
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_part);
    cudaFree(d_g);
    cudaFree(d_loss);
    return st;
}
