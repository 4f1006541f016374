// bd_policy.cu -- the learned direction policy: an fp32 8-32-32-2 MLP whose
// forward pass, backward pass and Adam update are hand-written kernels.
//
// The network replaces the alpha/beta rule of run_beamer
// (hybrid_bfs.cc:166-188) inside the persistent BFS kernel (decide_next in
// bd_bfs.cu evaluates it on the device: one warp per CTA, once per level,
// weights staged in shared memory).  Training
// data are per-level timings of forced top-down and forced bottom-up runs:
// both directions discover exactly the next BFS level, so the state after a
// step does not depend on the direction taken and the two timings at the
// same level form a counterfactual pair.  The label is the faster direction,
// the sample weight the time difference.
//
// Parameter vector (fp32, 1410 values): w1[32][8], b1[32], w2[32][32],
// b2[32], w3[2][32], b3[2] -- the first fields of PolicyBlob.
#include <cmath>
#include <cstring>
#include <vector>

#include "bd_bfs_device.cuh"
#include "bd_internal.h"

namespace bd {
namespace {

constexpr int kP = kPolicyParams;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kPolicyH * kPolicyIn;
constexpr int kOffW2 = kOffB1 + kPolicyH;
constexpr int kOffB2 = kOffW2 + kPolicyH * kPolicyH;
constexpr int kOffW3 = kOffB2 + kPolicyH;
constexpr int kOffB3 = kOffW3 + kPolicyOut * kPolicyH;
static_assert(kOffB3 + kPolicyOut == kP, "parameter layout");

constexpr int kTrainThreads = 256;

struct Hidden {
    float h1[kPolicyH];
    float h2[kPolicyH];
    float z[kPolicyOut];
};

__device__ __forceinline__ void mlp_forward(const float *P, const float *x, Hidden &h)
{
#pragma unroll 4
    for (int j = 0; j < kPolicyH; ++j) {
        float a = P[kOffB1 + j];
#pragma unroll
        for (int i = 0; i < kPolicyIn; ++i) { a += P[kOffW1 + j * kPolicyIn + i] * x[i]; }
        h.h1[j] = fmaxf(a, 0.f);
    }
#pragma unroll 2
    for (int k = 0; k < kPolicyH; ++k) {
        float a = P[kOffB2 + k];
#pragma unroll 8
        for (int j = 0; j < kPolicyH; ++j) { a += P[kOffW2 + k * kPolicyH + j] * h.h1[j]; }
        h.h2[k] = fmaxf(a, 0.f);
    }
#pragma unroll
    for (int o = 0; o < kPolicyOut; ++o) {
        float a = P[kOffB3 + o];
#pragma unroll 8
        for (int k = 0; k < kPolicyH; ++k) { a += P[kOffW3 + o * kPolicyH + k] * h.h2[k]; }
        h.z[o] = a;
    }
}

__global__ void policy_forward_kernel(const float *P, const float *X, int64_t n, float *logits)
{
    __shared__ float sp[kP];
    for (int i = threadIdx.x; i < kP; i += blockDim.x) { sp[i] = P[i]; }
    __syncthreads();
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n;
         s += (int64_t)gridDim.x * blockDim.x) {
        float x[kPolicyIn];
#pragma unroll
        for (int i = 0; i < kPolicyIn; ++i) { x[i] = X[s * kPolicyIn + i]; }
        Hidden h;
        mlp_forward(sp, x, h);
        logits[2 * s] = h.z[0];
        logits[2 * s + 1] = h.z[1];
    }
}

// Forward + backward of the weighted cross-entropy for one sample per
// thread; gradients are summed in shared memory, then once per block into
// the global gradient.  Scale: sum_i w_i CE_i * inv_wsum.
__global__ void policy_grad_kernel(const float *P, const float *X, const int32_t *label,
                                   const float *weight, int64_t n, float inv_wsum, float *grad,
                                   float *loss)
{
    __shared__ float sp[kP];
    __shared__ float sg[kP];
    __shared__ float sloss;
    for (int i = threadIdx.x; i < kP; i += blockDim.x) {
        sp[i] = P[i];
        sg[i] = 0.f;
    }
    if (threadIdx.x == 0) { sloss = 0.f; }
    __syncthreads();
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n;
         s += (int64_t)gridDim.x * blockDim.x) {
        float x[kPolicyIn];
#pragma unroll
        for (int i = 0; i < kPolicyIn; ++i) { x[i] = X[s * kPolicyIn + i]; }
        Hidden h;
        mlp_forward(sp, x, h);
        const int y = label[s];
        const float w = weight[s] * inv_wsum;
        const float zmax = fmaxf(h.z[0], h.z[1]);
        const float e0 = expf(h.z[0] - zmax), e1 = expf(h.z[1] - zmax);
        const float inv = 1.f / (e0 + e1);
        const float p0 = e0 * inv, p1 = e1 * inv;
        atomicAdd(&sloss, -w * logf(y ? p1 : p0));
        const float dz[2] = {(p0 - (y == 0 ? 1.f : 0.f)) * w, (p1 - (y == 1 ? 1.f : 0.f)) * w};
#pragma unroll
        for (int o = 0; o < kPolicyOut; ++o) { atomicAdd(&sg[kOffB3 + o], dz[o]); }
        float dh2[kPolicyH];
#pragma unroll 4
        for (int k = 0; k < kPolicyH; ++k) {
            atomicAdd(&sg[kOffW3 + k], dz[0] * h.h2[k]);
            atomicAdd(&sg[kOffW3 + kPolicyH + k], dz[1] * h.h2[k]);
            const float g = sp[kOffW3 + k] * dz[0] + sp[kOffW3 + kPolicyH + k] * dz[1];
            dh2[k] = h.h2[k] > 0.f ? g : 0.f;
        }
        float dh1[kPolicyH];
#pragma unroll 4
        for (int j = 0; j < kPolicyH; ++j) { dh1[j] = 0.f; }
        for (int k = 0; k < kPolicyH; ++k) {
            if (dh2[k] == 0.f) { continue; }
            atomicAdd(&sg[kOffB2 + k], dh2[k]);
#pragma unroll 8
            for (int j = 0; j < kPolicyH; ++j) {
                atomicAdd(&sg[kOffW2 + k * kPolicyH + j], dh2[k] * h.h1[j]);
                dh1[j] += sp[kOffW2 + k * kPolicyH + j] * dh2[k];
            }
        }
        for (int j = 0; j < kPolicyH; ++j) {
            const float g = h.h1[j] > 0.f ? dh1[j] : 0.f;
            if (g == 0.f) { continue; }
            atomicAdd(&sg[kOffB1 + j], g);
#pragma unroll
            for (int i = 0; i < kPolicyIn; ++i) { atomicAdd(&sg[kOffW1 + j * kPolicyIn + i], g * x[i]); }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kP; i += blockDim.x) {
        if (sg[i] != 0.f) { atomicAdd(&grad[i], sg[i]); }
    }
    if (threadIdx.x == 0 && loss) { atomicAdd(loss, sloss); }
}

// Adam (Kingma & Ba, 2015) with decoupled-from-nothing L2 term: g += wd * p.
__global__ void adam_kernel(float *P, const float *grad, float *m, float *v, int t, float lr,
                            float b1, float b2, float eps, float wd)
{
    const float c1 = 1.f - powf(b1, (float)t);
    const float c2 = 1.f - powf(b2, (float)t);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kP; i += gridDim.x * blockDim.x) {
        const float g = grad[i] + wd * P[i];
        const float mi = b1 * m[i] + (1.f - b1) * g;
        const float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

int blocks_for(int64_t n)
{
    int64_t b = (n + kTrainThreads - 1) / kTrainThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 4));
}

template <typename T>
struct DBuf {
    T *p = nullptr;
    ~DBuf() { if (p) { cudaFree(p); } }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * (n ? n : 1)); }
};

}  // namespace
}  // namespace bd

struct bd_bfs;
namespace bd {
// Defined in bd_bfs.cu: installs a PolicyBlob in the handle.
bd_status bfs_install_policy(bd_bfs *b, const PolicyBlob *blob);
}

namespace bd {

bd_status policy_blob(const float *params, const float *mean, const float *inv_std,
                      const float *lo, const float *hi, float margin, PolicyBlob *blob)
{
    if (!params || !mean || !inv_std || !(margin >= 0)) { return BD_ERR_INVALID; }
    memset(blob, 0, sizeof *blob);
    // params: w1[32][8], b1[32], w2[32][32], b2[32], w3[2][32], b3[2]
    const float *w1 = params;
    const float *b1 = w1 + kPolicyH * kPolicyIn;
    const float *w2 = b1 + kPolicyH;
    const float *b2 = w2 + kPolicyH * kPolicyH;
    const float *w3 = b2 + kPolicyH;
    const float *b3 = w3 + kPolicyOut * kPolicyH;
    for (int j = 0; j < kPolicyH; ++j) {
        for (int i = 0; i < kPolicyIn; ++i) { blob->w1t[i][j] = w1[j * kPolicyIn + i]; }
        for (int i = 0; i < kPolicyH; ++i) { blob->w2t[i][j] = w2[j * kPolicyH + i]; }
        blob->b1[j] = b1[j];
        blob->b2[j] = b2[j];
        blob->w3[0][j] = w3[j];
        blob->w3[1][j] = w3[kPolicyH + j];
    }
    blob->b3[0] = b3[0];
    blob->b3[1] = b3[1];
    memcpy(blob->mean, mean, sizeof(float) * kPolicyIn);
    memcpy(blob->inv_std, inv_std, sizeof(float) * kPolicyIn);
    for (int i = 0; i < kPolicyIn; ++i) {
        blob->lo[i] = lo ? lo[i] : -INFINITY;
        blob->hi[i] = hi ? hi[i] : INFINITY;
    }
    blob->margin = margin;
    return BD_OK;
}

}  // namespace bd

using namespace bd;

extern "C" {

bd_status bd_policy_forward(const float *params, const float *x, int64_t n, float *logits)
{
    if (!params || (!x && n) || (!logits && n) || n < 0) { return BD_ERR_INVALID; }
    if (n == 0) { return BD_OK; }
    BD_TRY(ensure_device());
    DBuf<float> dp, dx, dz;
    if (dp.alloc(kP) || dx.alloc(n * kPolicyIn) || dz.alloc(2 * n)) { return BD_ERR_OOM; }
    BD_CUDA(cudaMemcpy(dp.p, params, sizeof(float) * kP, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * n * kPolicyIn, cudaMemcpyHostToDevice));
    policy_forward_kernel<<<blocks_for(n), kTrainThreads>>>(dp.p, dx.p, n, dz.p);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaMemcpy(logits, dz.p, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost));
    return BD_OK;
}

bd_status bd_policy_loss_grad(const float *params, const float *x, const int32_t *label,
                              const float *weight, int64_t n, float *loss, float *grad)
{
    if (!params || !x || !label || !weight || n <= 0 || !grad) { return BD_ERR_INVALID; }
    double wsum = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (label[i] != 0 && label[i] != 1) { return BD_ERR_INVALID; }
        wsum += weight[i];
    }
    if (!(wsum > 0)) { return BD_ERR_INVALID; }
    BD_TRY(ensure_device());
    DBuf<float> dp, dx, dw, dg, dl;
    DBuf<int32_t> dy;
    if (dp.alloc(kP) || dx.alloc(n * kPolicyIn) || dw.alloc(n) || dg.alloc(kP) || dl.alloc(1) ||
        dy.alloc(n)) {
        return BD_ERR_OOM;
    }
    BD_CUDA(cudaMemcpy(dp.p, params, sizeof(float) * kP, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * n * kPolicyIn, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemcpy(dw.p, weight, sizeof(float) * n, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemcpy(dy.p, label, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemset(dg.p, 0, sizeof(float) * kP));
    BD_CUDA(cudaMemset(dl.p, 0, sizeof(float)));
    policy_grad_kernel<<<blocks_for(n), kTrainThreads>>>(dp.p, dx.p, dy.p, dw.p, n,
                                                        (float)(1.0 / wsum), dg.p, dl.p);
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaMemcpy(grad, dg.p, sizeof(float) * kP, cudaMemcpyDeviceToHost));
    if (loss) { BD_CUDA(cudaMemcpy(loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost)); }
    return BD_OK;
}

bd_status bd_policy_train(float *params, const float *x, const int32_t *label, const float *weight,
                          int64_t n, int32_t epochs, float lr, float weight_decay,
                          float *loss_history)
{
    if (!params || !x || !label || !weight || n <= 0 || epochs <= 0 || !(lr > 0)) {
        return BD_ERR_INVALID;
    }
    double wsum = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (label[i] != 0 && label[i] != 1) { return BD_ERR_INVALID; }
        wsum += weight[i];
    }
    if (!(wsum > 0)) { return BD_ERR_INVALID; }
    BD_TRY(ensure_device());
    DBuf<float> dp, dx, dw, dg, dm, dv, dl;
    DBuf<int32_t> dy;
    if (dp.alloc(kP) || dx.alloc(n * kPolicyIn) || dw.alloc(n) || dg.alloc(kP) || dm.alloc(kP) ||
        dv.alloc(kP) || dl.alloc(epochs) || dy.alloc(n)) {
        return BD_ERR_OOM;
    }
    BD_CUDA(cudaMemcpy(dp.p, params, sizeof(float) * kP, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * n * kPolicyIn, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemcpy(dw.p, weight, sizeof(float) * n, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemcpy(dy.p, label, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    BD_CUDA(cudaMemset(dm.p, 0, sizeof(float) * kP));
    BD_CUDA(cudaMemset(dv.p, 0, sizeof(float) * kP));
    BD_CUDA(cudaMemset(dl.p, 0, sizeof(float) * epochs));
    const float inv_wsum = (float)(1.0 / wsum);
    for (int t = 1; t <= epochs; ++t) {
        BD_CUDA(cudaMemsetAsync(dg.p, 0, sizeof(float) * kP));
        policy_grad_kernel<<<blocks_for(n), kTrainThreads>>>(dp.p, dx.p, dy.p, dw.p, n, inv_wsum,
                                                            dg.p, dl.p + (t - 1));
        adam_kernel<<<6, 256>>>(dp.p, dg.p, dm.p, dv.p, t, lr, 0.9f, 0.999f, 1e-8f, weight_decay);
    }
    BD_CUDA(cudaGetLastError());
    BD_CUDA(cudaDeviceSynchronize());
    BD_CUDA(cudaMemcpy(params, dp.p, sizeof(float) * kP, cudaMemcpyDeviceToHost));
    if (loss_history) {
        BD_CUDA(cudaMemcpy(loss_history, dl.p, sizeof(float) * epochs, cudaMemcpyDeviceToHost));
    }
    return BD_OK;
}

bd_status bd_bfs_set_policy(bd_bfs *b, const float *params, const float *mean,
                            const float *inv_std, const float *lo, const float *hi, float margin)
{
    if (!b) { return BD_ERR_INVALID; }
    // a margin of +inf: the rule decides every step, nothing is evaluated
    if (!params || isinf(margin)) { return bfs_install_policy(b, nullptr); }
    PolicyBlob blob;
    BD_TRY(policy_blob(params, mean, inv_std, lo, hi, margin, &blob));
    return bfs_install_policy(b, &blob);
}

}  // extern "C"
