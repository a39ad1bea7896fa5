// CSR SpMV building blocks with the reference's summation order.
//
// SparseMatricesCSR.jl's mul! (called at src/chebyshev.jl:47,165,179,287,305)
// accumulates each row over its stored entries in order: the three-argument
// form from zero, the five-argument form (beta == 1) term by term into y[row].
#pragma once

#include "hs_common.cuh"

namespace hsdev {

template <typename T>
struct AddOp {
    __device__ __forceinline__ T operator()(T a, T b) const { return add_rn(a, b); }
};
template <typename T>
struct SubOp {
    __device__ __forceinline__ T operator()(T a, T b) const { return sub_rn(a, b); }
};

// ---------------------------------------------------------------------------
// Block CSR-stream: a block of BR threads owns rows [row0, row0 + BR).  The
// products a_q * f(col_q) of all its entries are formed cooperatively (one
// entry per thread per pass: coalesced loads of ci/v and every gather in
// flight together) into shared memory, then thread t folds its row's products
// in storage order with `op` starting from `acc0`.  Bitwise the same sums as
// the sequential row loop.  When the block's entries exceed CAP, the threads
// fall back to folding straight from global memory (same arithmetic).
// ---------------------------------------------------------------------------
template <typename T, int BR, int CAP>
struct CsrStream {
    T prod[CAP];
    int32_t rs[BR + 1];
};

// Staged products per block: 8 per row at 256 rows, 32 per row at 128 rows.
template <int BR>
constexpr int stream_cap() { return BR >= 256 ? 2048 : 4096; }

// Entries per thread whose loads are issued before any of them is used.
constexpr int kU = 8;

// Returns (on every thread) the folded value of this thread's row, or acc0 for
// rows >= n.  `sh` is the block's shared staging area.  The product phase
// issues the loads of kU entries per thread (entry loads, then the dependent
// gathers) before using any of them, so a block keeps kU x BR entries in
// flight instead of one.
template <typename T, int BR, int CAP, typename F, typename Op>
__device__ __forceinline__ T csr_stream_fold(CsrStream<T, BR, CAP>& sh, int32_t n, const int32_t* __restrict__ rp,
                                             const int32_t* __restrict__ ci, const T* __restrict__ v,
                                             int64_t row0, T acc0, F f, Op op) {
    const int t = threadIdx.x;
    const int nrows = (int)min((int64_t)BR, (int64_t)n - row0);
    __syncthreads();   // previous use of sh is finished
    for (int i = t; i <= nrows; i += BR) sh.rs[i] = __ldg(rp + row0 + i);
    __syncthreads();
    const int32_t q0 = sh.rs[0];
    const int32_t cnt = sh.rs[nrows] - q0;
    T acc = acc0;
    if (cnt <= CAP) {
        for (int32_t base = 0; base < cnt; base += kU * BR) {
            int32_t c[kU];
            T a[kU], b[kU];
#pragma unroll
            for (int k = 0; k < kU; ++k) {
                const int32_t e = base + k * BR + t;
                if (e < cnt) {
                    c[k] = __ldg(ci + q0 + e);
                    a[k] = __ldg(v + q0 + e);
                }
            }
#pragma unroll
            for (int k = 0; k < kU; ++k)
                if (base + k * BR + t < cnt) b[k] = f(c[k]);
#pragma unroll
            for (int k = 0; k < kU; ++k) {
                const int32_t e = base + k * BR + t;
                if (e < cnt) sh.prod[e] = mul_rn(a[k], b[k]);
            }
        }
        __syncthreads();
        if (t < nrows) {
            const int32_t a = sh.rs[t] - q0, b = sh.rs[t + 1] - q0;
            for (int32_t e = a; e < b; ++e) acc = op(acc, sh.prod[e]);
        }
    } else if (t < nrows) {
        const int32_t a = sh.rs[t], b = sh.rs[t + 1];
        for (int32_t q = a; q < b; ++q) acc = op(acc, mul_rn(__ldg(v + q), f(__ldg(ci + q))));
    }
    return acc;
}

}  // namespace hsdev
