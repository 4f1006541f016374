// bd_policy.cuh -- the learned direction policy as the traversal kernels
// see it: the parameter blob and a one-warp forward pass.
#pragma once

#include <math.h>
#include <stdint.h>

namespace bd {

// 8-32-32-2 MLP, fp32.  The parameter vector the trainer uses is row-major
// (w1[32][8], b1, w2[32][32], b2, w3[2][32], b3); the traversal kernels keep
// the first two weight matrices transposed, so that lane j of the evaluating
// warp reads column j of consecutive rows (no shared-memory bank conflicts).
constexpr int kPolicyIn = 8;
constexpr int kPolicyH = 32;
constexpr int kPolicyOut = 2;
constexpr int kPolicyParams = kPolicyH * kPolicyIn + kPolicyH + kPolicyH * kPolicyH + kPolicyH +
                              kPolicyOut * kPolicyH + kPolicyOut;  // 1410
struct PolicyBlob {
    float w1t[kPolicyIn][kPolicyH];  // w1t[i][j] = w1[j][i]
    float b1[kPolicyH];
    float w2t[kPolicyH][kPolicyH];   // w2t[i][j] = w2[j][i]
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

// Raw feature i, in the order the trainer uses.  Every feature but the
// previous direction is a difference of two logarithms, so that graphs of
// any size share one range (a network trained on scales 16-24 is not
// outside its range at scale 26):
//   0  log2(1 + m_f) - log2(1 + m_u)     frontier degree sum over unexplored
//   1  log2(1 + frontier) - log2(1 + n)  frontier share of the vertices
//   2  log2(1 + m_u) - log2(1 + 2m)      unexplored share of the arcs
//   3  log2(1 + level)
//   4  log2(1 + m) - log2(1 + n)         average degree
//   5  previous direction (0 top-down / push, 1 bottom-up / pull)
//   6  log2(1 + previous step us) - log2(1 + m / 2^20)   time per M edges
//   7  log2(1 + m_f) - log2(1 + frontier) frontier average degree
// The lanes of a warp each pick their two arguments, then take two
// logarithms together (no divergent branches around the calls).
__device__ __forceinline__ float policy_feature(int i, long long frontier, long long frontier_edges,
                                                long long unexplored, int level, long long n,
                                                long long m, int prev_dir, long long prev_ns)
{
    float a = 0.f, b = 0.f;
    switch (i) {
        case 0: a = (float)frontier_edges; b = (float)unexplored; break;
        case 1: a = (float)frontier; b = (float)n; break;
        case 2: a = (float)unexplored; b = (float)(2 * m); break;
        case 3: a = (float)level; break;
        case 4: a = (float)m; b = (float)n; break;
        case 6: a = (float)prev_ns * 1e-3f; b = (float)m * (1.0f / 1048576.0f); break;
        case 7: a = (float)frontier_edges; b = (float)frontier; break;
        default: break;
    }
    a = fmaxf(a, 0.f);
    b = fmaxf(b, 0.f);
    const float d = log2f(1.0f + a) - log2f(1.0f + b);
    return i == 5 ? (float)prev_dir : d;
}

// Feature 0 alone (thread 0, before the network is woken): the policy is
// only consulted where feature 0 lies in its trusted range, the band in
// which the trainer saw the best direction differ from the rule's.
__device__ __forceinline__ bool policy_in_band(const PolicyBlob *w, long long frontier_edges,
                                               long long unexplored)
{
    const float f0 = log2f(1.0f + (float)(frontier_edges > 0 ? frontier_edges : 0)) -
                     log2f(1.0f + (float)(unexplored > 0 ? unexplored : 0));
    return f0 >= w->lo[0] && f0 <= w->hi[0];
}

// Forward pass by the 32 lanes of one warp (lane j owns hidden unit j;
// lanes 0-7 compute the features, activations move by shuffles).  Returns,
// in every lane, the logit gap (bottom-up minus top-down), or NaN when a
// feature lies outside the trusted range.  w may point to shared or global
// memory.
__device__ __forceinline__ float policy_gap_warp(const PolicyBlob *w, long long frontier,
                                                 long long frontier_edges, long long unexplored,
                                                 int level, long long n, long long m,
                                                 int prev_dir, long long prev_ns)
{
    const unsigned full = 0xFFFFFFFFu;
    const int j = threadIdx.x & 31;
    float x = 0.f;
    bool ok = true;
    if (j < kPolicyIn) {
        const float f = policy_feature(j, frontier, frontier_edges, unexplored, level, n, m,
                                       prev_dir, prev_ns);
        ok = f >= w->lo[j] && f <= w->hi[j];
        x = (f - w->mean[j]) * w->inv_std[j];
    }
    // outside the trusted range the rule decides: skip the network
    if (!__all_sync(full, ok)) { return nanf(""); }
    float a1 = w->b1[j];
#pragma unroll
    for (int i = 0; i < kPolicyIn; ++i) { a1 += w->w1t[i][j] * __shfl_sync(full, x, i); }
    const float h1 = fmaxf(a1, 0.f);
    float a2 = w->b2[j], a2b = 0.f;  // two chains: half the dependent adds
#pragma unroll
    for (int i = 0; i < kPolicyH; i += 2) {
        a2 += w->w2t[i][j] * __shfl_sync(full, h1, i);
        a2b += w->w2t[i + 1][j] * __shfl_sync(full, h1, i + 1);
    }
    const float h2 = fmaxf(a2 + a2b, 0.f);
    float o0 = w->w3[0][j] * h2, o1 = w->w3[1][j] * h2;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        o0 += __shfl_xor_sync(full, o0, d);
        o1 += __shfl_xor_sync(full, o1, d);
    }
    return (o1 + w->b3[1]) - (o0 + w->b3[0]);
}

}  // namespace bd
