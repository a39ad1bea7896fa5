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

// ---- compensated ("Dot2") accumulation ---------------------------------
// Ogita, Rump & Oishi (2005), Accurate sum and dot product: a sum carried as
// an unevaluated pair (s, c) with error-free transformations.  The result is
// as accurate as a dot computed in twice the working precision, so it rounds to
// the same double whatever the summation order (up to ties at the 2^-106
// level).  The Krylov drivers use it so that their trajectories reproduce the
// CPU restatement, which uses the same accumulation.
struct DD {
    double s, c;
};

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

// acc += a*b: TwoProduct (exact via fma) then TwoSum, errors into acc.c
__device__ __forceinline__ void dd_add_prod(DD& acc, double a, double b) {
    const double p = __dmul_rn(a, b);
    const double pe = __fma_rn(a, b, -p);
    double t, q;
    two_sum(acc.s, p, t, q);
    acc.s = t;
    acc.c = __dadd_rn(acc.c, __dadd_rn(q, pe));
}

__device__ __forceinline__ DD dd_add(DD a, DD b) {
    double t, q;
    two_sum(a.s, b.s, t, q);
    return DD{t, __dadd_rn(__dadd_rn(a.c, b.c), q)};
}

__device__ __forceinline__ double dd_value(DD v) { return __dadd_rn(v.s, v.c); }

__device__ __forceinline__ DD warp_dd(DD v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        DD w{__shfl_xor_sync(0xffffffffu, v.s, o), __shfl_xor_sync(0xffffffffu, v.c, o)};
        v = dd_add(v, w);
    }
    return v;
}

// Block-wide compensated sum; result valid on thread 0.
__device__ __forceinline__ DD block_dd(DD v) {
    __shared__ double shs[32], shc[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_dd(v);
    __syncthreads();
    if (lane == 0) {
        shs[warp] = v.s;
        shc[warp] = v.c;
    }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? DD{shs[threadIdx.x], shc[threadIdx.x]} : DD{0.0, 0.0};
    if (warp == 0) v = warp_dd(v);
    return v;
}

// block_dd with thread 0's result broadcast to every thread of the block.
__device__ __forceinline__ DD block_dd_all(DD v) {
    __shared__ double bs, bc;
    v = block_dd(v);
    if (threadIdx.x == 0) {
        bs = v.s;
        bc = v.c;
    }
    __syncthreads();
    v = DD{bs, bc};
    __syncthreads();   // bs/bc may be reused by the next call
    return v;
}

inline int red_blocks(int64_t n) {
    int64_t b = (n + kRedThreads - 1) / kRedThreads;
    return (int)(b < 1 ? 1 : (b > kRedMaxBlocks ? kRedMaxBlocks : b));
}

}  // namespace hsdev
