// bd_policy.cuh -- the learned direction policy as the traversal kernels
// see it: the parameter blob and a one-warp forward pass.
#pragma once

#include <math.h>
#include <stdint.h>

namespace bd {

// 8-32-32-2 MLP, fp32, row-major weights.
constexpr int kPolicyIn = 8;
constexpr int kPolicyH = 32;
constexpr int kPolicyOut = 2;
constexpr int kPolicyParams = kPolicyH * kPolicyIn + kPolicyH + kPolicyH * kPolicyH + kPolicyH +
                              kPolicyOut * kPolicyH + kPolicyOut;  // 1410
struct PolicyBlob {
    float w1[kPolicyH][kPolicyIn];
    float b1[kPolicyH];
    float w2[kPolicyH][kPolicyH];
    float b2[kPolicyH];
    float w3[kPolicyOut][kPolicyH];
    float b3[kPolicyOut];
    float mean[kPolicyIn];   // feature standardisation
    float inv_std[kPolicyIn];
    float lo[kPolicyIn];     // raw-feature range the policy trusts; outside
    float hi[kPolicyIn];     // it the rule decides
    float margin;            // |logit gap| below which the rule decides
    float pad[3];
};

__device__ __forceinline__ float policy_log2p1(double x) { return (float)log2(1.0 + (x > 0 ? x : 0)); }

// Raw features, in the order the trainer uses: log2(1 + frontier vertices),
// log2(1 + frontier degree sum), log2(1 + unexplored degree sum), level,
// log2(1 + n), log2(1 + m), previous direction, log2(1 + previous step us).
__device__ __forceinline__ void policy_features(float *f, long long frontier,
                                                long long frontier_edges, long long unexplored,
                                                int level, long long n, long long m,
                                                int prev_dir, long long prev_ns)
{
    f[0] = policy_log2p1((double)frontier);
    f[1] = policy_log2p1((double)frontier_edges);
    f[2] = policy_log2p1((double)unexplored);
    f[3] = (float)level;
    f[4] = policy_log2p1((double)n);
    f[5] = policy_log2p1((double)m);
    f[6] = (float)prev_dir;
    f[7] = policy_log2p1((double)prev_ns * 1e-3);
}

// Forward pass by the 32 lanes of one warp (lane j owns hidden unit j).
// feat and h1 live in shared memory.  Returns, in every lane, the logit gap
// (bottom-up minus top-down), or NaN when a feature lies outside the
// trusted range.
__device__ __forceinline__ float policy_gap_warp(const PolicyBlob *w, const float *feat, float *h1)
{
    const int j = threadIdx.x & 31;
    bool trusted = true;
#pragma unroll
    for (int i = 0; i < kPolicyIn; ++i) {
        trusted = trusted && feat[i] >= w->lo[i] && feat[i] <= w->hi[i];
    }
    float a1 = w->b1[j];
#pragma unroll
    for (int i = 0; i < kPolicyIn; ++i) { a1 += w->w1[j][i] * ((feat[i] - w->mean[i]) * w->inv_std[i]); }
    h1[j] = fmaxf(a1, 0.f);
    __syncwarp();
    float a2 = w->b2[j];
#pragma unroll 8
    for (int i = 0; i < kPolicyH; ++i) { a2 += w->w2[j][i] * h1[i]; }
    const float h2 = fmaxf(a2, 0.f);
    float o0 = w->w3[0][j] * h2, o1 = w->w3[1][j] * h2;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        o0 += __shfl_xor_sync(0xFFFFFFFFu, o0, d);
        o1 += __shfl_xor_sync(0xFFFFFFFFu, o1, d);
    }
    __syncwarp();
    const float gap = (o1 + w->b3[1]) - (o0 + w->b3[0]);
    return trusted ? gap : nanf("");
}

}  // namespace bd
