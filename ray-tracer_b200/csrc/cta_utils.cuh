// cta_utils.cuh -- block-level scans and reductions used by the build kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rtb
{

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) { x += y; }
    }
    return x;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t x)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, o); }
    return x;
}

// Exclusive scan of one value per thread across a block of BLOCK threads (multiple of 32).
// `sh` needs BLOCK/32 + 1 words. Returns the exclusive prefix; *total receives the block sum.
template <int BLOCK>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total)
{
    constexpr int W = BLOCK / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t x = warp_incl_scan(v);
    if (lane == 31) { sh[warp] = x; }
    __syncthreads();
    if (warp == 0)
    {
        uint32_t w = lane < W ? sh[lane] : 0u;
        w = warp_incl_scan(w);
        if (lane < W) { sh[lane] = w; }
    }
    __syncthreads();
    const uint32_t base = warp > 0 ? sh[warp - 1] : 0u;
    const uint32_t tot = sh[W - 1];
    __syncthreads();
    if (total) { *total = tot; }
    return base + x - v;
}

template <int BLOCK>
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* sh)
{
    uint32_t t;
    block_excl_scan<BLOCK>(v, sh, &t);
    return t;
}

} // namespace rtb
