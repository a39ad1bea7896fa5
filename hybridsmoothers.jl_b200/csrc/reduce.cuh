// Deterministic FP64 reductions: each block reduces its slice with a fixed
// shuffle tree into partials[blockIdx.x]; a single-block finalize kernel sums
// the partials in a fixed order.  Same inputs -> same bits, whatever else runs
// on the GPU (the serving path relies on this).
#pragma once

#include "hs_common.cuh"

namespace hsdev {

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 1184;  // 148 SMs x 8

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum with a fixed tree; result valid on thread 0.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
    if (warp == 0) v = warp_sum(v);
    return v;
}

// partials[0..nparts) -> *out, fixed order.  One block of kRedThreads.
// If sqrt_out, *out = sqrt(sum).
static __global__ void finalize_sum_kernel(const double* __restrict__ partials, int nparts, double* __restrict__ out,
                                           int sqrt_out) {
    double v = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) v = __dadd_rn(v, partials[i]);
    v = block_sum(v);
    if (threadIdx.x == 0) *out = sqrt_out ? sqrt(v) : v;
}

// Dot product partials of a and b over [0, n).
template <typename TA, typename TB>
__global__ void dot_partials_kernel(const TA* __restrict__ a, const TB* __restrict__ b, int64_t n,
                                    double* __restrict__ partials) {
    double v = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v = __dadd_rn(v, __dmul_rn((double)a[i], (double)b[i]));
    v = block_sum(v);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
}

inline int red_blocks(int64_t n) {
    int64_t b = (n + kRedThreads - 1) / kRedThreads;
    return (int)(b < 1 ? 1 : (b > kRedMaxBlocks ? kRedMaxBlocks : b));
}

}  // namespace hsdev
