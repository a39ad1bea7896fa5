// CSR SpMV building blocks with the reference's summation order.
//
// SparseMatricesCSR.jl's mul! (called at src/chebyshev.jl:47,165,179,287,305)
// accumulates each row over its stored entries in order: the three-argument
// form from zero, the five-argument form (beta == 1) term by term into y[row].
// A row is handled by a sub-warp of LPR lanes: the lanes load LPR consecutive
// entries (coalesced), form their products, and the sub-warp leader folds
// them in storage order through shuffles, so the sum is the sequential one.
#pragma once

#include "hs_common.cuh"

namespace hsdev {

// Ordered fold of per-lane values `v` (valid where m < cnt) into acc on the
// sub-warp leader; op(acc, v) is applied in lane order 0..LPR-1.
template <int LPR, typename T, typename Op>
__device__ __forceinline__ T ordered_fold(T acc, T v, int cnt, int sub_base, Op op) {
    const int sublane = threadIdx.x & (LPR - 1);
#pragma unroll
    for (int m = 0; m < LPR; ++m) {
        const T pm = __shfl_sync(0xffffffffu, v, sub_base + m);
        if (sublane == 0 && m < cnt) acc = op(acc, pm);
    }
    return acc;
}

// Row sum_j a_ij * f(j) in storage order, accumulated into acc0 with `op`.
// Returns the result on the sub-warp leader.  All lanes of the warp must
// call it (shuffles are warp-wide); rows >= n contribute nothing.
template <int LPR, typename T, typename F, typename Op>
__device__ __forceinline__ T row_fold(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                      const T* __restrict__ v, int64_t row, bool valid, T acc0, F f, Op op,
                                      int max_chunks) {
    const int lane = threadIdx.x & 31;
    const int sublane = lane & (LPR - 1);
    const int sub_base = lane - sublane;
    int32_t p0 = 0, p1 = 0;
    if (valid) {
        p0 = __ldg(rp + row);
        p1 = __ldg(rp + row + 1);
    }
    T acc = acc0;
    // every lane iterates the warp-uniform chunk count
    for (int c = 0; c < max_chunks; ++c) {
        const int32_t base = p0 + c * LPR;
        const int cnt = valid ? min(LPR, p1 - base) : 0;
        T prod = T(0);
        if (sublane < cnt) {
            const int32_t q = base + sublane;
            prod = mul_rn(__ldg(v + q), f(__ldg(ci + q)));
        }
        acc = ordered_fold<LPR>(acc, prod, cnt, sub_base, op);
    }
    return acc;
}

template <typename T>
struct AddOp {
    __device__ __forceinline__ T operator()(T a, T b) const { return add_rn(a, b); }
};
template <typename T>
struct SubOp {
    __device__ __forceinline__ T operator()(T a, T b) const { return sub_rn(a, b); }
};

// Number of LPR-chunks of the longest row in this warp's rows.
template <int LPR>
__device__ __forceinline__ int warp_max_chunks(const int32_t* __restrict__ rp, int64_t row, bool valid) {
    int c = 0;
    if (valid && (threadIdx.x & (LPR - 1)) == 0) {
        const int len = __ldg(rp + row + 1) - __ldg(rp + row);
        c = (len + LPR - 1) / LPR;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
    return c;
}

}  // namespace hsdev
