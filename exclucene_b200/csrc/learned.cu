// Learned position models: storage and device residency. The training and
// leaf-fit kernels are added in learned_train.cu.
#include <cuda_runtime.h>

#include <vector>

#include "excl_device.cuh"
#include "runtime.h"

namespace excl {

struct ModelSet {
    std::vector<float> root;     // kRootStride floats per model
    std::vector<ModelHdr> hdr;
    std::vector<Leaf> leaves;
    float *d_root = nullptr;
    ModelHdr *d_hdr = nullptr;
    Leaf *d_leaves = nullptr;
    int device = 0;
};

ModelView model_view(const ModelSet *m) {
    ModelView v;
    if (m) {
        v.root = m->d_root;
        v.hdr = m->d_hdr;
        v.leaves = m->d_leaves;
    }
    return v;
}

void models_free(ModelSet *m) {
    if (!m) return;
    cudaFree(m->d_root);
    cudaFree(m->d_hdr);
    cudaFree(m->d_leaves);
    delete m;
}

int models_upload(excl_ctx *ctx, excl_index *ix) {
    ModelSet *m = ix->models;
    if (!m || m->hdr.empty()) return EXCL_OK;
    cudaFree(m->d_root);
    cudaFree(m->d_hdr);
    cudaFree(m->d_leaves);
    m->d_root = nullptr;
    m->d_hdr = nullptr;
    m->d_leaves = nullptr;
    int st = cuda_status(ctx, cudaMalloc((void **)&m->d_root, m->root.size() * 4), "model alloc");
    if (!st) st = cuda_status(ctx, cudaMalloc((void **)&m->d_hdr, m->hdr.size() * sizeof(ModelHdr)), "model alloc");
    if (!st) st = cuda_status(ctx, cudaMalloc((void **)&m->d_leaves, m->leaves.size() * sizeof(Leaf)), "model alloc");
    if (!st)
        st = cuda_status(ctx, cudaMemcpy(m->d_root, m->root.data(), m->root.size() * 4, cudaMemcpyHostToDevice), "up");
    if (!st)
        st = cuda_status(ctx, cudaMemcpy(m->d_hdr, m->hdr.data(), m->hdr.size() * sizeof(ModelHdr), cudaMemcpyHostToDevice),
                         "up");
    if (!st)
        st = cuda_status(
            ctx, cudaMemcpy(m->d_leaves, m->leaves.data(), m->leaves.size() * sizeof(Leaf), cudaMemcpyHostToDevice), "up");
    m->device = ctx->device;
    return st;
}

}  // namespace excl
