// bd_device_util.cuh -- small device helpers shared by the traversal kernels.
#pragma once

#include <stdint.h>

namespace bd {
namespace dev {

constexpr unsigned kFullMask = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Arrival at a grid barrier: orders every write the CTA made before it (the
// CTA synchronised with __syncthreads first) ahead of the increment.
__device__ __forceinline__ void red_release_add64(unsigned long long *p, unsigned long long v)
{
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (long long)t;
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T x)
{
    const int lane = lane_id();
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T y = __shfl_up_sync(kFullMask, x, d);
        if (lane >= d) { x += y; }
    }
    return x;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T x)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) { x += __shfl_xor_sync(kFullMask, x, d); }
    return x;
}

__device__ __forceinline__ unsigned long long warp_or(unsigned long long x)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) { x |= __shfl_xor_sync(kFullMask, x, d); }
    return x;
}

// OR of the values of lanes below this one.
__device__ __forceinline__ unsigned long long warp_excl_or(unsigned long long x)
{
    const int lane = lane_id();
    unsigned long long incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        unsigned long long y = __shfl_up_sync(kFullMask, incl, d);
        if (lane >= d) { incl |= y; }
    }
    unsigned long long excl = __shfl_up_sync(kFullMask, incl, 1);
    return lane == 0 ? 0ull : excl;
}

}  // namespace dev
}  // namespace bd
