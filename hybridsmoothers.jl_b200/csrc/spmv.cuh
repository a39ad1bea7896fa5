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
// Warp CSR-stream: a warp owns 32 consecutive rows [row0, row0 + 32).  Its
// entries are processed in windows of WCAP: the products a_q * f(col_q) of a
// window are formed by all 32 lanes (coalesced ci/v loads, KU entries per
// lane issued before their gathers) into the warp's private shared buffer,
// and lane l then folds the part of row row0+l that lies in the window, in
// storage order, continuing from the previous window.  Only __syncwarp
// between phases: warps never wait for each other, so each SM keeps many
// warps' loads in flight.  Bitwise the sequential row sums, any row length.
// Every lane of the warp must call it; rows >= n get acc0 back.
// ---------------------------------------------------------------------------
constexpr int kWarpCap = 256;   // products per window (2 KB of FP64 per warp)
constexpr int kWarpKU = 4;      // entries per lane per load round

// The row pointers of a lane's row in the 32-row chunk at row0 (0, 0 past n).
struct RowPtrs {
    int32_t ra, rb;
};
__device__ __forceinline__ RowPtrs load_rowptrs(int32_t n, const int32_t* __restrict__ rp, int64_t row0) {
    const int64_t r = row0 + (threadIdx.x & 31);
    RowPtrs p{0, 0};
    if (r < n) {
        p.ra = __ldg(rp + r);
        p.rb = __ldg(rp + r + 1);
    }
    return p;
}

template <typename T, typename F, typename Op>
__device__ __forceinline__ T csr_warp_fold_rp(T* __restrict__ wbuf, int32_t n, RowPtrs rpp,
                                              const int32_t* __restrict__ ci, const T* __restrict__ v, int64_t row0,
                                              T acc0, F f, Op op);

template <typename T, typename F, typename Op>
__device__ __forceinline__ T csr_warp_fold(T* __restrict__ wbuf, int32_t n, const int32_t* __restrict__ rp,
                                           const int32_t* __restrict__ ci, const T* __restrict__ v, int64_t row0,
                                           T acc0, F f, Op op) {
    return csr_warp_fold_rp(wbuf, n, load_rowptrs(n, rp, row0), ci, v, row0, acc0, f, op);
}

// csr_warp_fold with the chunk's row pointers already loaded (load_rowptrs).
template <typename T, typename F, typename Op>
__device__ __forceinline__ T csr_warp_fold_rp(T* __restrict__ wbuf, int32_t n, RowPtrs rpp,
                                              const int32_t* __restrict__ ci, const T* __restrict__ v, int64_t row0,
                                              T acc0, F f, Op op) {
    const int lane = threadIdx.x & 31;
    const int64_t r = row0 + lane;
    const bool valid = r < n;
    const int nrows = (int)min((int64_t)32, (int64_t)n - row0);
    const int32_t ra = rpp.ra, rb = rpp.rb;
    const int32_t q0 = __shfl_sync(0xffffffffu, ra, 0);
    const int32_t q1 = __shfl_sync(0xffffffffu, rb, nrows - 1);
    T acc = acc0;
    for (int32_t base = q0; base < q1; base += kWarpCap) {
        const int32_t cnt = min(kWarpCap, q1 - base);
        for (int32_t k0 = 0; k0 < cnt; k0 += 32 * kWarpKU) {
            int32_t c[kWarpKU];
            T a[kWarpKU], b[kWarpKU];
#pragma unroll
            for (int k = 0; k < kWarpKU; ++k) {
                const int32_t e = k0 + k * 32 + lane;
                if (e < cnt) {
                    c[k] = __ldg(ci + base + e);
                    a[k] = __ldg(v + base + e);
                }
            }
#pragma unroll
            for (int k = 0; k < kWarpKU; ++k)
                if (k0 + k * 32 + lane < cnt) b[k] = f(c[k]);
#pragma unroll
            for (int k = 0; k < kWarpKU; ++k) {
                const int32_t e = k0 + k * 32 + lane;
                if (e < cnt) wbuf[e] = mul_rn(a[k], b[k]);
            }
        }
        __syncwarp();
        if (valid) {
            const int32_t lo = max(ra, base), hi = min(rb, base + cnt);
            for (int32_t e = lo; e < hi; ++e) acc = op(acc, wbuf[e - base]);
        }
        __syncwarp();
    }
    return acc;
}

// ---- 32-row slices ---------------------------------------------------------
// A matrix in 32-row slices: slice s holds w_s entries per row (w_s its
// longest row) stored column by column ([k][row]) from soff[s], so lane r
// reads entry k of its row at soff[s] + 32 k + r -- coalesced, with no row
// pointers and no window in shared memory.  A row's entries keep their
// storage order and its padding entries (column -1) follow them and are
// skipped, so every fold is the CSR fold's sequence of operations exactly.

// ent[s] = 32 * w_s for s < nslices, ent[nslices] = 0 (exclusive-scan input).
__global__ void slice_width_kernel(int32_t n, int64_t nslices, const int32_t* __restrict__ rp,
                                   int64_t* __restrict__ ent);

// The entries of each slice (soff: the exclusive scan of slice_width_kernel);
// padding entries get column -1.
template <typename T>
__global__ void slice_fill_kernel(int32_t n, int64_t nslices, const int32_t* __restrict__ rp,
                                  const int32_t* __restrict__ ci, const T* __restrict__ v,
                                  const int64_t* __restrict__ soff, int32_t* __restrict__ scol,
                                  T* __restrict__ sval) {
    const int lane = threadIdx.x & 31;
    for (int64_t sl = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; sl < nslices;
         sl += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t o = soff[sl];
        const int32_t w = (int32_t)((soff[sl + 1] - o) / 32);
        const int64_t row = sl * 32 + lane;
        const int32_t q0 = row < n ? rp[row] : 0, len = row < n ? rp[row + 1] - q0 : 0;
        for (int32_t k = 0; k < w; ++k) {
            const bool real = k < len;
            scol[o + 32 * (int64_t)k + lane] = real ? ci[q0 + k] : -1;
            sval[o + 32 * (int64_t)k + lane] = real ? v[q0 + k] : T(0);
        }
    }
}

// Fold of row (32 s + lane) for the slice with entries [o0, o1):
// acc = op(acc, v_k * fx(c_k)) over the row's entries in storage order, as
// csr_warp_fold does; eight entries of the row in flight at a time.
template <typename T, typename F, typename Op>
__device__ __forceinline__ T slice_row_fold(int64_t o0, int64_t o1, const int32_t* __restrict__ scol,
                                            const T* __restrict__ sval, T acc, F fx, Op op) {
    constexpr int KU = 8;
    const int lane = threadIdx.x & 31;
    const int32_t w = (int32_t)((o1 - o0) / 32);
    const int32_t* __restrict__ cp = scol + o0 + lane;
    const T* __restrict__ vp = sval + o0 + lane;
    for (int32_t j = 0; j < w; j += KU) {
        int32_t c[KU];
        T a[KU], b[KU];
#pragma unroll
        for (int u = 0; u < KU; ++u) {
            c[u] = j + u < w ? __ldg(cp + 32 * (j + u)) : -1;
            a[u] = j + u < w ? __ldg(vp + 32 * (j + u)) : T(0);
        }
#pragma unroll
        for (int u = 0; u < KU; ++u) b[u] = c[u] >= 0 ? fx(c[u]) : T(0);
#pragma unroll
        for (int u = 0; u < KU; ++u)
            if (c[u] >= 0) acc = op(acc, mul_rn(a[u], b[u]));
    }
    return acc;
}

// Row (32 s + lane) of A times x: the storage-order sum from +0.
template <typename F>
__device__ __forceinline__ double slice_row_sum(int64_t o0, int64_t o1, const int32_t* __restrict__ scol,
                                                const double* __restrict__ sval, F fx) {
    return slice_row_fold(o0, o1, scol, sval, 0.0, fx, AddOp<double>());
}

}  // namespace hsdev
