// Sparse matrix (mul!) and Chebyshev smoothers for B200 (sm_100a).
//
// Reference: src/chebyshev.jl of HybridSmoothers.jl v0.1.4 and the CSR mul!
// of SparseMatricesCSR.jl that it calls.
//
// Fusion.  Each Chebyshev step is ONE kernel that applies the vector update
// and the SpMV that follows it:
//   4th kind, step k (chebyshev.jl:172-181):
//     z_k = a_k z_{k-1} + (b_k l1inv) r_{k-1};  x += z_k;  r_k = r_{k-1} - A z_k
//     The SpMV needs z_k at the neighbours; each lane recomputes z_k[j] from
//     z_{k-1}[j], r_{k-1}[j], l1inv[j] with the same operations, so the value
//     is bitwise the one row j stores.  z and r are double-buffered.
//   1st kind, step k < degree (:298-319):
//     x += z_{k-1};  r -= (l1inv * (A z_{k-1})) * inv_rho;
//     z_k = c1 z_{k-1} + c2 r           (z double-buffered)
// Every sum is in storage order with separately rounded multiply/add (see
// spmv.cuh), so FP64 results are bitwise the reference's order of operations
// at a given rho.  rho comes from an FP64 power iteration on the device whose
// norm is a fixed-order parallel sum (the reference's BLAS nrm2 order is
// library-specific), so rho matches the reference to rounding.
#include <algorithm>
#include <mutex>
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "internal.cuh"
#include "reduce.cuh"
#include "spmv.cuh"

using hsdev::AddOp;
using hsdev::SubOp;

// ---------------------------------------------------------------------------
// Device CSR matrix
// ---------------------------------------------------------------------------
struct hs_matrix_s {
    int32_t n = 0;
    int64_t nnz = 0;
    int32_t dtype = HS_F64;
    int32_t* rp = nullptr;
    int32_t* ci = nullptr;
    void* v = nullptr;
    // FP64 copy in 32-row slices (spmv.cuh), built at the first PCG solve
    int64_t* soff = nullptr;
    int32_t* scol = nullptr;
    void* sval = nullptr;      // values in the matrix type
    int64_t bytes = 0;
    bool stream_ordered = false;   // buffers from cudaMallocAsync
    cudaStream_t alloc_stream = nullptr;
};

namespace hsm {

inline size_t dsize(int dt) { return dt == HS_F64 ? 8 : 4; }

// Host CSR (row-wise) arrays from an hs_sparse, values as double.
void host_csr(const hs_sparse* A, std::vector<int32_t>& rp, std::vector<int32_t>& ci, std::vector<double>& v) {
    const int32_t n = A->n;
    auto val = [&](int64_t q) -> double {
        return A->dtype == HS_F64 ? static_cast<const double*>(A->val)[q] : (double)static_cast<const float*>(A->val)[q];
    };
    if (A->format == HS_CSR) {
        rp.assign(A->ptr, A->ptr + n + 1);
        ci.assign(A->idx, A->idx + A->nnz);
        v.resize(A->nnz);
        for (int64_t q = 0; q < A->nnz; ++q) v[q] = val(q);
        return;
    }
    rp.assign(n + 1, 0);
    for (int64_t q = 0; q < A->nnz; ++q) rp[A->idx[q] + 1]++;
    for (int32_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
    std::vector<int32_t> cur(rp.begin(), rp.end() - 1);
    ci.resize(A->nnz);
    v.resize(A->nnz);
    for (int32_t col = 0; col < n; ++col)
        for (int32_t q = A->ptr[col]; q < A->ptr[col + 1]; ++q) {
            const int32_t r = A->idx[q];
            ci[cur[r]] = col;
            v[cur[r]] = val(q);
            cur[r]++;
        }
}

int validate(const hs_sparse* A) {
    if (!A || A->n <= 0 || !A->ptr) return hs::set_error(HS_ERR_ARG, "invalid matrix descriptor");
    if (A->format != HS_CSC && A->format != HS_CSR) return hs::set_error(HS_ERR_ARG, "unknown matrix format");
    if (A->dtype != HS_F64 && A->dtype != HS_F32) return hs::set_error(HS_ERR_ARG, "unknown value type");
    if (A->nnz < 0 || A->nnz > INT32_MAX || A->ptr[0] != 0 || A->ptr[A->n] != A->nnz)
        return hs::set_error(HS_ERR_ARG, "pointer array must start at 0 and end at nnz");
    if (A->nnz > 0 && (!A->idx || !A->val)) return hs::set_error(HS_ERR_ARG, "matrix arrays are NULL");
    for (int32_t c = 0; c < A->n; ++c) {
        if (A->ptr[c + 1] < A->ptr[c]) return hs::set_error(HS_ERR_ARG, "pointer array is not monotone");
        for (int32_t q = A->ptr[c]; q < A->ptr[c + 1]; ++q) {
            if (A->idx[q] < 0 || A->idx[q] >= A->n) return hs::set_error(HS_ERR_ARG, "index out of range");
            if (q > A->ptr[c] && A->idx[q - 1] >= A->idx[q])
                return hs::set_error(HS_ERR_ARG, "indices must be strictly ascending");
        }
    }
    return HS_OK;
}

int matrix_from_host(const std::vector<int32_t>& rp, const std::vector<int32_t>& ci, const std::vector<double>& v,
                     int32_t dtype, cudaStream_t st, hs_matrix** out) {
    hs_matrix* M = new hs_matrix();
    M->n = (int32_t)rp.size() - 1;
    M->nnz = (int64_t)ci.size();
    M->dtype = dtype;
    const size_t es = dsize(dtype);
    cudaError_t e;
    if ((e = cudaMalloc(&M->rp, sizeof(int32_t) * rp.size())) != cudaSuccess ||
        (e = cudaMalloc(&M->ci, sizeof(int32_t) * std::max<size_t>(1, ci.size()))) != cudaSuccess ||
        (e = cudaMalloc(&M->v, es * std::max<size_t>(1, v.size()))) != cudaSuccess) {
        cudaFree(M->rp);
        cudaFree(M->ci);
        cudaFree(M->v);
        delete M;
        return hs::cuda_error(e, "cudaMalloc (matrix)");
    }
    M->bytes = (int64_t)(sizeof(int32_t) * (rp.size() + ci.size()) + es * v.size());
    HS_CUDA(cudaMemcpyAsync(M->rp, rp.data(), sizeof(int32_t) * rp.size(), cudaMemcpyHostToDevice, st));
    HS_CUDA(cudaMemcpyAsync(M->ci, ci.data(), sizeof(int32_t) * ci.size(), cudaMemcpyHostToDevice, st));
    if (dtype == HS_F64) {
        HS_CUDA(cudaMemcpyAsync(M->v, v.data(), es * v.size(), cudaMemcpyHostToDevice, st));
        HS_CUDA(cudaStreamSynchronize(st));
    } else {
        std::vector<float> f(v.size());
        for (size_t q = 0; q < v.size(); ++q) f[q] = (float)v[q];
        HS_CUDA(cudaMemcpyAsync(M->v, f.data(), es * f.size(), cudaMemcpyHostToDevice, st));
        HS_CUDA(cudaStreamSynchronize(st));
    }
    *out = M;
    return HS_OK;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;
// The plain SpMV with five resident CTAs per SM (48 registers): it is
// latency-bound, and the extra warps measured 10-12 % faster FP64 SpMVs than
// the unbounded register allocation (4 CTAs); six spill.  The fused Chebyshev
// steps keep their registers (the same cap made them 22 % slower).
constexpr int kWarpMinBlocks = 5;

// Every SpMV-shaped kernel below runs the warp CSR-stream of spmv.cuh
// (csr_warp_fold): a warp owns 32 consecutive rows at a time and warps stride
// over the matrix; a CTA is kThreads threads with one product window per warp.
#define HS_WARP_SHARED(T) __shared__ T wbuf[kThreads / 32][hsdev::kWarpCap]
#define HS_WARP_ROWS_LOOP                                                                                   \
    const int warp_ = threadIdx.x >> 5;                                                                       \
    for (int64_t row0 = ((int64_t)blockIdx.x * (kThreads / 32) + warp_) * 32; row0 < n;                       \
         row0 += (int64_t)gridDim.x * kThreads)
#define HS_WARP_FOLD(acc0, f, op) hsdev::csr_warp_fold(wbuf[warp_], n, rp, ci, v, row0, acc0, f, op)
// The same fold over the matrix's 32-row slices when the kernel has them
// (soff non-null): the same operations in the same order.
#define HS_ROW_FOLD(acc0, f, op)                                                                        \
    (soff ? hsdev::slice_row_fold(soff[row0 >> 5], soff[(row0 >> 5) + 1], scol, sval, acc0, f, op) \
          : HS_WARP_FOLD(acc0, f, op))
#define HS_SLICE_PARAMS(T) \
    const int64_t *__restrict__ soff, const int32_t *__restrict__ scol, const T *__restrict__ sval

// MODE 0: y = A x; MODE 1: y = y - A x (term by term); MODE 2: y = beta y + sum (a x) alpha.
template <typename T, int MODE>
__global__ void __launch_bounds__(kThreads, kWarpMinBlocks) spmv_kernel(int32_t n, const int32_t* __restrict__ rp,
                                                        const int32_t* __restrict__ ci, const T* __restrict__ v,
                                                        const T* __restrict__ x, T* __restrict__ y, T alpha, T beta) {
    HS_WARP_SHARED(T);
    auto fx = [&](int32_t j) { return __ldg(x + j); };
    HS_WARP_ROWS_LOOP {
        const int64_t r = row0 + (threadIdx.x & 31);
        const bool valid = r < n;
        T acc;
        if (MODE == 0) {
            acc = HS_WARP_FOLD(T(0), fx, AddOp<T>());
        } else if (MODE == 1) {
            acc = HS_WARP_FOLD(valid ? y[r] : T(0), fx, SubOp<T>());
        } else {
            T a0 = T(0);
            if (valid && beta != T(0)) a0 = (beta == T(1)) ? y[r] : mul_rn(y[r], beta);
            auto op = [alpha](T a, T p) { return add_rn(a, mul_rn(p, alpha)); };
            acc = HS_WARP_FOLD(a0, fx, op);
        }
        if (valid) y[r] = acc;
    }
}

// The same three forms over the matrix's 32-row slices (FP64): the folds of
// spmv_kernel, operation for operation.
template <int MODE>
__global__ void __launch_bounds__(kThreads, 4) spmv_sliced_kernel(int32_t n, const int64_t* __restrict__ soff,
                                                              const int32_t* __restrict__ scol,
                                                              const double* __restrict__ sval,
                                                              const double* __restrict__ x, double* __restrict__ y,
                                                              double alpha, double beta) {
    auto fx = [&](int32_t j) { return __ldg(x + j); };
    const int64_t nsl = ((int64_t)n + 31) / 32;
    const int64_t stride = (int64_t)gridDim.x * (kThreads / 32);
    for (int64_t sl = (int64_t)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); sl < nsl; sl += stride) {
        const int64_t r = sl * 32 + (threadIdx.x & 31);
        const bool valid = r < n;
        const int64_t o0 = soff[sl], o1 = soff[sl + 1];
        double acc;
        if (MODE == 0) {
            acc = hsdev::slice_row_fold(o0, o1, scol, sval, 0.0, fx, AddOp<double>());
        } else if (MODE == 1) {
            acc = hsdev::slice_row_fold(o0, o1, scol, sval, valid ? y[r] : 0.0, fx, SubOp<double>());
        } else {
            double a0 = 0.0;
            if (valid && beta != 0.0) a0 = (beta == 1.0) ? y[r] : __dmul_rn(y[r], beta);
            auto op = [alpha](double a, double p) { return __dadd_rn(a, __dmul_rn(p, alpha)); };
            acc = hsdev::slice_row_fold(o0, o1, scol, sval, a0, fx, op);
        }
        if (valid) y[r] = acc;
    }
}

// l1inv[i] = 1 / sum_j |a_ij| (storage order), FP64: _l1_rowsum (chebyshev.jl:27-36)
__global__ void l1inv_kernel(int32_t n, const int32_t* __restrict__ rp, const double* __restrict__ v,
                             double* __restrict__ l1inv) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int32_t q = rp[i]; q < rp[i + 1]; ++q) s = __dadd_rn(s, fabs(v[q]));
        l1inv[i] = __ddiv_rn(1.0, s);
    }
}

template <typename TA, typename TB>
__global__ void convert_kernel(const TA* __restrict__ a, TB* __restrict__ b, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (TB)a[i];
}

template <typename T>
__global__ void fill_kernel(T* __restrict__ a, int64_t n, T value) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = value;
}

// Power iteration step (chebyshev.jl:46-51): w = l1inv .* (A v); partial sum
// of w.^2 per CTA (grid <= partials capacity).
__global__ void __launch_bounds__(kThreads) power_spmv_kernel(int32_t n, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci,
                                                              const double* __restrict__ v,
                                                              const double* __restrict__ vin,
                                                              const double* __restrict__ l1inv,
                                                              double* __restrict__ w, double* __restrict__ partials,
                                                              const int* __restrict__ stop) {
    if (*stop) return;
    HS_WARP_SHARED(double);
    auto fx = [&](int32_t j) { return __ldg(vin + j); };
    double ss = 0.0;
    HS_WARP_ROWS_LOOP {
        const int64_t r = row0 + (threadIdx.x & 31);
        const double acc = HS_WARP_FOLD(0.0, fx, AddOp<double>());
        if (r < n) {
            const double wi = __dmul_rn(acc, l1inv[r]);
            w[r] = wi;
            ss = __dadd_rn(ss, __dmul_rn(wi, wi));
        }
    }
    ss = hsdev::block_sum(ss);
    if (threadIdx.x == 0) partials[blockIdx.x] = ss;
}

// rho = sqrt(sum partials); stop once rho == 0 (iszero(rho) && break).
__global__ void power_finalize_kernel(const double* __restrict__ partials, int nparts, double* __restrict__ rho,
                                      int* __restrict__ stop) {
    if (*stop) return;
    double v = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) v = __dadd_rn(v, partials[i]);
    v = hsdev::block_sum(v);
    if (threadIdx.x == 0) {
        const double r = sqrt(v);
        *rho = r;
        if (r == 0.0) *stop = 1;
    }
}

__global__ void power_normalize_kernel(int32_t n, const double* __restrict__ w, const double* __restrict__ rho,
                                       double* __restrict__ vout, const int* __restrict__ stop) {
    if (*stop) return;
    const double r = *rho;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        vout[i] = __ddiv_rn(w[i], r);
}

// Lanczos operator w = dm .* (A (dm .* v)), dm = sqrt(l1inv).
__global__ void __launch_bounds__(kThreads) lanczos_op_kernel(int32_t n, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci,
                                                              const double* __restrict__ v,
                                                              const double* __restrict__ vin,
                                                              const double* __restrict__ dm, double* __restrict__ w) {
    HS_WARP_SHARED(double);
    auto fx = [&](int32_t j) { return __dmul_rn(__ldg(dm + j), __ldg(vin + j)); };
    HS_WARP_ROWS_LOOP {
        const int64_t r = row0 + (threadIdx.x & 31);
        const double acc = HS_WARP_FOLD(0.0, fx, AddOp<double>());
        if (r < n) w[r] = __dmul_rn(dm[r], acc);
    }
}

__global__ void lanczos_update_kernel(int32_t n, double* __restrict__ w, const double* __restrict__ v,
                                      const double* __restrict__ vprev, double alpha, double beta) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        w[i] = w[i] - alpha * v[i] - beta * vprev[i];
}

__global__ void scale_kernel(int32_t n, const double* __restrict__ w, double inv, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = w[i] * inv;
}

__global__ void sqrt_kernel(int32_t n, const double* __restrict__ a, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = sqrt(a[i]);
}

// ---- Chebyshev 4th kind ----------------------------------------------------
// r = b - A x (chebyshev.jl:165-167), z = 0 (:170)
template <typename T>
__global__ void __launch_bounds__(kThreads) cheb4_init_kernel(int32_t n, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci, const T* __restrict__ v,
                                                              HS_SLICE_PARAMS(T), const T* __restrict__ x, const T* __restrict__ b,
                                                              T* __restrict__ r, T* __restrict__ z) {
    HS_WARP_SHARED(T);
    auto fx = [&](int32_t j) { return __ldg(x + j); };
    HS_WARP_ROWS_LOOP {
        const int64_t i = row0 + (threadIdx.x & 31);
        const T ax = HS_ROW_FOLD(T(0), fx, AddOp<T>());
        if (i < n) {
            r[i] = sub_rn(b[i], ax);
            z[i] = T(0);
        }
    }
}

// x = 0 start: A*0 sums to +0, so r = b - (+0) = b exactly; z = 0; x = 0.
template <typename T, typename IO>
__global__ void cheb4_init_zero_kernel(int32_t n, const IO* __restrict__ b, T* __restrict__ r, T* __restrict__ z,
                                       T* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        r[i] = (T)b[i];
        z[i] = T(0);
        x[i] = T(0);
    }
}

// One fused step (chebyshev.jl:176-179 with kernel :132-139).
template <typename T>
__global__ void __launch_bounds__(kThreads) cheb4_step_kernel(int32_t n, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci, const T* __restrict__ v,
                                                              HS_SLICE_PARAMS(T), const T* __restrict__ l1inv, T ak, T bk,
                                                              const T* __restrict__ z_old, const T* __restrict__ r_old,
                                                              T* __restrict__ z_new, T* __restrict__ r_new,
                                                              T* __restrict__ x) {
    HS_WARP_SHARED(T);
    auto zk = [&](int32_t j) {
        return add_rn(mul_rn(ak, __ldg(z_old + j)), mul_rn(mul_rn(bk, __ldg(l1inv + j)), __ldg(r_old + j)));
    };
    HS_WARP_ROWS_LOOP {
        const int64_t i = row0 + (threadIdx.x & 31);
        const bool valid = i < n;
        const T acc = HS_ROW_FOLD(valid ? r_old[i] : T(0), zk, SubOp<T>());
        if (valid) {
            const T zi = zk((int32_t)i);
            z_new[i] = zi;
            x[i] = add_rn(x[i], zi);
            r_new[i] = acc;
        }
    }
}

// ---- Chebyshev 1st kind ----------------------------------------------------
// tmp = A x; r = (l1inv (b - tmp)) inv_rho; z = c0 r   (chebyshev.jl:287-293, :237-244)
template <typename T>
__global__ void __launch_bounds__(kThreads) cheb1_init_kernel(int32_t n, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci, const T* __restrict__ v,
                                                              HS_SLICE_PARAMS(T), const T* __restrict__ x, const T* __restrict__ b,
                                                              const T* __restrict__ l1inv, T inv_rho, T c0,
                                                              T* __restrict__ r, T* __restrict__ z) {
    HS_WARP_SHARED(T);
    auto fx = [&](int32_t j) { return __ldg(x + j); };
    HS_WARP_ROWS_LOOP {
        const int64_t i = row0 + (threadIdx.x & 31);
        const T tmp = HS_ROW_FOLD(T(0), fx, AddOp<T>());
        if (i < n) {
            const T ri = mul_rn(mul_rn(l1inv[i], sub_rn(b[i], tmp)), inv_rho);
            r[i] = ri;
            z[i] = mul_rn(c0, ri);
        }
    }
}

template <typename T, typename IO>
__global__ void cheb1_init_zero_kernel(int32_t n, const IO* __restrict__ b, const T* __restrict__ l1inv, T inv_rho,
                                       T c0, T* __restrict__ r, T* __restrict__ z, T* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T ri = mul_rn(mul_rn(l1inv[i], (T)b[i]), inv_rho);
        r[i] = ri;
        z[i] = mul_rn(c0, ri);
        x[i] = T(0);
    }
}

// x += z_old; r -= (l1inv (A z_old)) inv_rho; z_new = c1 z_old + c2 r   (:300-316)
template <typename T>
__global__ void __launch_bounds__(kThreads) cheb1_step_kernel(int32_t n, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci, const T* __restrict__ v,
                                                              HS_SLICE_PARAMS(T), const T* __restrict__ l1inv, T inv_rho, T c1, T c2,
                                                              const T* __restrict__ z_old, T* __restrict__ z_new,
                                                              T* __restrict__ r, T* __restrict__ x) {
    HS_WARP_SHARED(T);
    auto fz = [&](int32_t j) { return __ldg(z_old + j); };
    HS_WARP_ROWS_LOOP {
        const int64_t i = row0 + (threadIdx.x & 31);
        const T tmp = HS_ROW_FOLD(T(0), fz, AddOp<T>());
        if (i < n) {
            const T zo = z_old[i];
            x[i] = add_rn(x[i], zo);
            const T rn = sub_rn(r[i], mul_rn(mul_rn(l1inv[i], tmp), inv_rho));
            r[i] = rn;
            z_new[i] = add_rn(mul_rn(c1, zo), mul_rn(c2, rn));
        }
    }
}

template <typename T>
__global__ void axpy_one_kernel(int32_t n, T* __restrict__ x, const T* __restrict__ z) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = add_rn(x[i], z[i]);
}

// One CTA per kThreads rows (a warp per 32): the block scheduler streams them
// through the SMs.
inline int grid_rows(int64_t n) {
    const int64_t blocks = (n + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, INT32_MAX));
}
inline int grid_elems(int64_t n) {
    const int64_t b = (n + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)hs::num_sms() * 16));
}

template <typename T>
int spmv_t(const hs_matrix* M, const void* x, void* y, double alpha, double beta, cudaStream_t st) {
    const int g = grid_rows(M->n);
    if (sizeof(T) == 8) {
        // FP64: the sliced copy (built here unless the stream is being captured)
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(st, &cs);
        const int64_t* so = M->soff;
        const int32_t* sc = M->scol;
        const void* svv = M->sval;
        if (!so && cs == cudaStreamCaptureStatusNone) {
            if (int rc = hs::matrix_slices(const_cast<hs_matrix*>(M), st, &so, &sc, &svv)) return rc;
        }
        const double* sv = static_cast<const double*>(svv);
        if (so) {
            const double* xx = static_cast<const double*>(x);
            double* yy = static_cast<double*>(y);
            if (alpha == 1.0 && beta == 0.0)
                spmv_sliced_kernel<0><<<g, kThreads, 0, st>>>(M->n, so, sc, sv, xx, yy, 1.0, 0.0);
            else if (alpha == -1.0 && beta == 1.0)
                spmv_sliced_kernel<1><<<g, kThreads, 0, st>>>(M->n, so, sc, sv, xx, yy, -1.0, 1.0);
            else
                spmv_sliced_kernel<2><<<g, kThreads, 0, st>>>(M->n, so, sc, sv, xx, yy, alpha, beta);
            HS_LAUNCH_CHECK("spmv_sliced_kernel");
            return HS_OK;
        }
    }
    const T* v = static_cast<const T*>(M->v);
    const T* xx = static_cast<const T*>(x);
    T* yy = static_cast<T*>(y);
    if (alpha == 1.0 && beta == 0.0) {
        spmv_kernel<T, 0><<<g, kThreads, 0, st>>>(M->n, M->rp, M->ci, v, xx, yy, T(1), T(0));
    } else if (alpha == -1.0 && beta == 1.0) {
        spmv_kernel<T, 1><<<g, kThreads, 0, st>>>(M->n, M->rp, M->ci, v, xx, yy, T(-1), T(1));
    } else {
        spmv_kernel<T, 2><<<g, kThreads, 0, st>>>(M->n, M->rp, M->ci, v, xx, yy, (T)alpha, (T)beta);
    }
    HS_LAUNCH_CHECK("spmv_kernel");
    return HS_OK;
}

}  // namespace hsm

// Internal entry used by the Krylov drivers.
namespace hs {
int matrix_spmv(const hs_matrix* M, const void* x, void* y, double alpha, double beta, cudaStream_t st) {
    return M->dtype == HS_F64 ? hsm::spmv_t<double>(M, x, y, alpha, beta, st)
                              : hsm::spmv_t<float>(M, x, y, alpha, beta, st);
}
// The FP64 matrix in 32-row slices, built once (on stream st; one wait for
// the entry count) and kept with the matrix.
int matrix_slices(hs_matrix* M, cudaStream_t st, const int64_t** soff, const int32_t** scol, const void** sval) {
    if (!M->soff) {
        const size_t es = M->dtype == HS_F64 ? 8 : 4;
        const int32_t n = M->n;
        const int64_t nsl = ((int64_t)n + 31) / 32;
        const bool so = M->stream_ordered;
        auto alloc = [&](void** p, size_t bytes) -> cudaError_t {
            return so ? cudaMallocAsync(p, bytes ? bytes : 16, st) : cudaMalloc(p, bytes ? bytes : 16);
        };
        auto release = [&](void* p) {
            if (!p) return;
            if (so)
                cudaFreeAsync(p, st);
            else
                cudaFree(p);
        };
        int64_t* ent = nullptr;
        int64_t* off = nullptr;
        void* tmp = nullptr;
        size_t tbytes = 0;
        int64_t total = 0;
        cudaError_t e;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((32 * (nsl + 1) + 255) / 256, 8192));
        if ((e = alloc((void**)&ent, sizeof(int64_t) * (size_t)(nsl + 1))) ||
            (e = alloc((void**)&off, sizeof(int64_t) * (size_t)(nsl + 1))))
            goto fail;
        hsdev::slice_width_kernel<<<grid, 256, 0, st>>>(n, nsl, M->rp, ent);
        hs::count_launch();
        if ((e = cub::DeviceScan::ExclusiveSum(nullptr, tbytes, ent, off, nsl + 1, st)) ||
            (e = alloc(&tmp, tbytes)) || (e = cub::DeviceScan::ExclusiveSum(tmp, tbytes, ent, off, nsl + 1, st)) ||
            (e = cudaMemcpyAsync(&total, off + nsl, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st)))
            goto fail;
        release(tmp);
        tmp = nullptr;
        release(ent);
        ent = nullptr;
        if ((e = alloc((void**)&M->scol, sizeof(int32_t) * (size_t)total)) ||
            (e = alloc((void**)&M->sval, es * (size_t)total)))
            goto fail;
        if (M->dtype == HS_F64)
            hsdev::slice_fill_kernel<double><<<grid, 256, 0, st>>>(n, nsl, M->rp, M->ci, static_cast<const double*>(M->v),
                                                                   off, M->scol, static_cast<double*>(M->sval));
        else
            hsdev::slice_fill_kernel<float><<<grid, 256, 0, st>>>(n, nsl, M->rp, M->ci, static_cast<const float*>(M->v),
                                                                  off, M->scol, static_cast<float*>(M->sval));
        hs::count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) goto fail;
        M->soff = off;
        M->bytes += (int64_t)(8 * (nsl + 1) + (4 + (int64_t)es) * total);
        goto done;
    fail:
        release(tmp);
        release(ent);
        release(off);
        release(M->scol);
        release(M->sval);
        M->scol = nullptr;
        M->sval = nullptr;
        return hs::cuda_error(e, "sliced matrix copy");
    done:;
    }
    *soff = M->soff;
    *scol = M->scol;
    *sval = M->sval;
    return HS_OK;
}

int matrix_n(const hs_matrix* M) { return M->n; }
int64_t matrix_nnz(const hs_matrix* M) { return M->nnz; }
void matrix_arrays(const hs_matrix* M, const int32_t** rp, const int32_t** ci, const void** v, int* dtype) {
    *rp = M->rp;
    *ci = M->ci;
    *v = M->v;
    *dtype = M->dtype;
}
}  // namespace hs

// ---------------------------------------------------------------------------
// Chebyshev handle
// ---------------------------------------------------------------------------
struct hs_cheb_s {
    int32_t n = 0, kind = 4, degree = 4, eig = 0, sdt = HS_F64;
    double rho = 1, rho_power = 0, lmin = 0, lmax = 0, astar = 0;
    hs_matrix* A = nullptr;      // smoother-precision CSR
    void* l1inv = nullptr;       // smoother precision
    void* w[6] = {nullptr};      // r0 r1 z0 z1 xbuf bbuf
    int64_t bytes = 0;
};

namespace hsm {

void destroy_matrix(hs_matrix* M, cudaStream_t free_stream = nullptr) {
    if (!M) return;
    void* ptrs[] = {M->rp, M->ci, M->v, M->soff, M->scol, M->sval};
    for (void* q : ptrs) {
        if (!q) continue;
        if (M->stream_ordered)
            cudaFreeAsync(q, free_stream ? free_stream : M->alloc_stream);
        else
            cudaFree(q);
    }
    delete M;
}

void destroy_cheb(hs_cheb* S) {
    if (!S) return;
    destroy_matrix(S->A);
    cudaFree(S->l1inv);
    for (void* p : S->w) cudaFree(p);
    delete S;
}

double astar(int k) {
    // _cheb1_astar (chebyshev.jl:81-89): bisection on x = sqrt(a*), 60 steps.
    double lo = 1e-10, hi = 1.0 - 1e-10;
    for (int it = 0; it < 60; ++it) {
        const double mid = (lo + hi) / 2;
        const double phi = 8.0 * k * std::pow(1 - mid * mid, 2 * k) +
                           mid * (std::pow(1 - mid, 4 * k) - std::pow(1 + mid, 4 * k));
        if (phi > 0) lo = mid; else hi = mid;
    }
    const double m = (lo + hi) / 2;
    return m * m;
}

// Eigenvalue bounds of the Lanczos tridiagonal (alpha, beta) by Sturm bisection.
void tridiag_extremes(const std::vector<double>& a, const std::vector<double>& b, double& lmin, double& lmax) {
    const int k = (int)a.size();
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < k; ++i) {
        const double r = (i > 0 ? std::fabs(b[i - 1]) : 0) + (i + 1 < k ? std::fabs(b[i]) : 0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    auto count_below = [&](double x) {
        int c = 0;
        double d = 1.0;
        for (int i = 0; i < k; ++i) {
            const double bb = i > 0 ? b[i - 1] * b[i - 1] : 0.0;
            d = a[i] - x - (i > 0 ? bb / d : 0.0);
            if (d == 0.0) d = -1e-300;
            if (d < 0) ++c;
        }
        return c;
    };
    auto kth = [&](int idx) {
        double l = lo, h = hi;
        for (int it = 0; it < 200; ++it) {
            const double m = 0.5 * (l + h);
            if (count_below(m) > idx) h = m; else l = m;
        }
        return 0.5 * (l + h);
    };
    lmin = kth(0);
    lmax = kth(k - 1);
}

template <typename T>
int cheb_smooth_t(hs_cheb* S, T* x, const void* b, int io, bool x_is_zero, cudaStream_t st) {
    const int32_t n = S->n;
    const hs_matrix* M = S->A;
    const T* v = static_cast<const T*>(M->v);
    const int64_t* so = M->soff;   // the sliced copy (built with the smoother)
    const int32_t* sc = M->scol;
    const T* sv = static_cast<const T*>(M->sval);
    const T* l1 = static_cast<const T*>(S->l1inv);
    T* r[2] = {static_cast<T*>(S->w[0]), static_cast<T*>(S->w[1])};
    T* z[2] = {static_cast<T*>(S->w[2]), static_cast<T*>(S->w[3])};
    const int g = grid_rows(n), ge = grid_elems(n);
    if (S->kind == 4) {
        if (x_is_zero) {
            if (io == HS_F64)
                cheb4_init_zero_kernel<T, double><<<ge, kThreads, 0, st>>>(n, static_cast<const double*>(b), r[0], z[0], x);
            else
                cheb4_init_zero_kernel<T, float><<<ge, kThreads, 0, st>>>(n, static_cast<const float*>(b), r[0], z[0], x);
            HS_LAUNCH_CHECK("cheb4_init_zero_kernel");
        } else {
            cheb4_init_kernel<T><<<g, kThreads, 0, st>>>(
                                        n, M->rp, M->ci, v, so, sc, sv, x, static_cast<const T*>(b), r[0], z[0]);
            HS_LAUNCH_CHECK("cheb4_init_kernel");
        }
        int cur = 0;
        for (int k = 1; k <= S->degree; ++k) {
            const T ak = (T)((double)(2 * k - 3) / (double)(2 * k + 1));
            const T bk = (T)((double)(8 * k - 4) / ((double)(2 * k + 1) * S->rho));
            cheb4_step_kernel<T><<<g, kThreads, 0, st>>>(
                                        n, M->rp, M->ci, v, so, sc, sv, l1, ak, bk, z[cur], r[cur], z[cur ^ 1], r[cur ^ 1], x);
            HS_LAUNCH_CHECK("cheb4_step_kernel");
            cur ^= 1;
        }
        return HS_OK;
    }
    // 1st kind; scalars in double, rounded where they meet vectors.
    const double a = S->astar;
    const T inv_rho = (T)(1.0 / S->rho);
    const T c0 = (T)(2.0 / (1.0 + a));
    if (x_is_zero) {
        if (io == HS_F64)
            cheb1_init_zero_kernel<T, double><<<ge, kThreads, 0, st>>>(n, static_cast<const double*>(b), l1, inv_rho, c0,
                                                                       r[0], z[0], x);
        else
            cheb1_init_zero_kernel<T, float><<<ge, kThreads, 0, st>>>(n, static_cast<const float*>(b), l1, inv_rho, c0,
                                                                      r[0], z[0], x);
        HS_LAUNCH_CHECK("cheb1_init_zero_kernel");
    } else {
        cheb1_init_kernel<T><<<g, kThreads, 0, st>>>(
                                    n, M->rp, M->ci, v, so, sc, sv, x, static_cast<const T*>(b), l1, inv_rho, c0, r[0], z[0]);
        HS_LAUNCH_CHECK("cheb1_init_kernel");
    }
    double rho_s = (1.0 - a) / (1.0 + a);
    int cur = 0;
    for (int k = 1; k <= S->degree; ++k) {
        if (k < S->degree) {
            const double rho_new = 1.0 / (2.0 * (1.0 + a) / (1.0 - a) - rho_s);
            const T c1 = (T)(rho_new * rho_s);
            const T c2 = (T)(4.0 * rho_new / (1.0 - a));
            cheb1_step_kernel<T><<<g, kThreads, 0, st>>>(
                                        n, M->rp, M->ci, v, so, sc, sv, l1, inv_rho, c1, c2, z[cur], z[cur ^ 1], r[0], x);
            HS_LAUNCH_CHECK("cheb1_step_kernel");
            cur ^= 1;
            rho_s = rho_new;
        } else {
            axpy_one_kernel<T><<<ge, kThreads, 0, st>>>(n, x, z[cur]);
            HS_LAUNCH_CHECK("axpy_one_kernel");
        }
    }
    return HS_OK;
}

}  // namespace hsm

namespace {
int matrix_create_impl(const hs_sparse* A, int32_t dtype, void* stream, hs_matrix** out, bool stream_ordered) {
    if (!out) return hs::set_error(HS_ERR_ARG, "out is NULL");
    *out = nullptr;
    int rc = hsm::validate(A);
    if (rc) return rc;
    if (dtype != HS_F64 && dtype != HS_F32) return hs::set_error(HS_ERR_ARG, "unknown dtype");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    hs_matrix* M = new hs_matrix();
    M->stream_ordered = stream_ordered;
    M->alloc_stream = st;
    M->n = A->n;
    M->nnz = A->nnz;
    M->dtype = dtype;
    const size_t es = hsm::dsize(dtype);
    cudaError_t e;
    auto alloc = [&](void** p, size_t bytes) {
        return stream_ordered ? cudaMallocAsync(p, bytes, st) : cudaMalloc(p, bytes);
    };
    if ((e = alloc((void**)&M->rp, sizeof(int32_t) * (M->n + 1))) != cudaSuccess ||
        (e = alloc((void**)&M->ci, sizeof(int32_t) * std::max<int64_t>(1, M->nnz))) != cudaSuccess ||
        (e = alloc(&M->v, es * std::max<int64_t>(1, M->nnz))) != cudaSuccess) {
        hsm::destroy_matrix(M);
        return hs::cuda_error(e, "cudaMalloc (matrix)");
    }
    M->bytes = (int64_t)(sizeof(int32_t) * (M->n + 1 + M->nnz) + es * M->nnz);
    // A CSC input is transposed on the device (stable: rows keep ascending columns).
    rc = hs::csr_from_host(A, dtype, M->rp, M->ci, M->v, st);
    if (!rc && !stream_ordered) {   // stream-ordered callers order their own use
        const cudaError_t se = cudaStreamSynchronize(st);
        if (se != cudaSuccess) rc = hs::cuda_error(se, "hs_matrix_create");
    }
    if (rc) {
        hsm::destroy_matrix(M);
        return rc;
    }
    *out = M;
    return HS_OK;
}

}  // namespace

namespace hs {
// Matrix whose buffers come from the stream-ordered pool on `st`, released
// with matrix_destroy_async (no device synchronisation).
int matrix_create_async(const hs_sparse* A, int32_t dtype, cudaStream_t st, hs_matrix** out) {
    return matrix_create_impl(A, dtype, st, out, true);
}
void matrix_destroy_async(hs_matrix* M, cudaStream_t st) { hsm::destroy_matrix(M, st); }
}  // namespace hs

extern "C" {

int hs_matrix_create(const hs_sparse* A, int32_t dtype, void* stream, hs_matrix** out) {
    return matrix_create_impl(A, dtype, stream, out, false);
}

int hs_matrix_spmv(hs_matrix* A, const void* x, void* y, double alpha, double beta, void* stream) {
    if (!A || !x || !y) return hs::set_error(HS_ERR_ARG, "hs_matrix_spmv: NULL argument");
    return hs::matrix_spmv(A, x, y, alpha, beta, static_cast<cudaStream_t>(stream));
}

int hs_matrix_destroy(hs_matrix* A) {
    if (A) cudaDeviceSynchronize();
    hsm::destroy_matrix(A);
    return HS_OK;
}

int hs_cheb_create(const hs_sparse* A, int32_t kind, int32_t degree, int32_t eig, int32_t smoother_dtype, void* stream,
                   hs_cheb** out) {
    if (!out) return hs::set_error(HS_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (kind != 1 && kind != 4) return hs::set_error(HS_ERR_ARG, "kind must be 1 or 4");
    if (degree < 1) return hs::set_error(HS_ERR_ARG, "degree must be at least 1");
    if (eig != HS_EIG_POWER && eig != HS_EIG_LANCZOS) return hs::set_error(HS_ERR_ARG, "unknown eig mode");
    if (smoother_dtype != HS_F64 && smoother_dtype != HS_F32) return hs::set_error(HS_ERR_ARG, "unknown dtype");
    int rc = hsm::validate(A);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<int32_t> rp, ci;
    std::vector<double> v;
    hsm::host_csr(A, rp, ci, v);   // SparseMatrixCSR(A_csc) (chebyshev.jl:144, :261)
    hs_cheb* S = new hs_cheb();
    S->n = A->n;
    S->kind = kind;
    S->degree = degree;
    S->eig = eig;
    S->sdt = smoother_dtype;
    hs_matrix* M64 = nullptr;
    if ((rc = hsm::matrix_from_host(rp, ci, v, HS_F64, st, &M64))) {
        hsm::destroy_cheb(S);
        return rc;
    }
    const int32_t n = S->n;
    double *l1inv = nullptr, *vv = nullptr, *ww = nullptr, *partials = nullptr, *rho_d = nullptr;
    int* stop = nullptr;
    auto fail = [&](int code) {
        cudaFree(l1inv); cudaFree(vv); cudaFree(ww); cudaFree(partials); cudaFree(rho_d); cudaFree(stop);
        hsm::destroy_matrix(M64);
        hsm::destroy_cheb(S);
        return code;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&l1inv, 8 * (size_t)n)) || (e = cudaMalloc(&vv, 8 * (size_t)n)) ||
        (e = cudaMalloc(&ww, 8 * (size_t)n)) || (e = cudaMalloc(&partials, 8 * hsdev::kRedMaxBlocks)) ||
        (e = cudaMalloc(&rho_d, 8)) || (e = cudaMalloc(&stop, sizeof(int))))
        return fail(hs::cuda_error(e, "cudaMalloc (chebyshev setup)"));
    const int ge = hsm::grid_elems(n);
    hsm::l1inv_kernel<<<ge, hsm::kThreads, 0, st>>>(n, M64->rp, static_cast<const double*>(M64->v), l1inv);
    hs::count_launch();
    // power iteration, chebyshev.jl:40-54
    hsm::fill_kernel<double><<<ge, hsm::kThreads, 0, st>>>(vv, n, 1.0 / std::sqrt((double)n));
    hs::count_launch();
    cudaMemsetAsync(stop, 0, sizeof(int), st);
    // The power-iteration SpMV writes one partial per block: keep its grid within
    // the partials buffer (kRedMaxBlocks); the kernel strides over row blocks.
    const int gr = std::min(hsm::grid_rows(n), hsdev::kRedMaxBlocks);
    for (int it = 0; it < 50; ++it) {
        hsm::power_spmv_kernel<<<gr, hsm::kThreads, 0, st>>>(
                                      n, M64->rp, M64->ci, static_cast<const double*>(M64->v), vv, l1inv, ww, partials,
                                      stop);
        hsm::power_finalize_kernel<<<1, hsdev::kRedThreads, 0, st>>>(partials, gr, rho_d, stop);
        hsm::power_normalize_kernel<<<ge, hsm::kThreads, 0, st>>>(n, ww, rho_d, vv, stop);
        hs::count_launch(3);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(hs::cuda_error(e, "power iteration"));
    if ((e = cudaMemcpyAsync(&S->rho_power, rho_d, 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
        return fail(hs::cuda_error(e, "power iteration"));
    S->rho = S->rho_power;
    if (eig == HS_EIG_LANCZOS) {
        // Lanczos on dm A dm (similar to M^-1 A, M = diag(l1)), 40 steps, FP64.
        double *dm = nullptr, *vp = nullptr, *sc = nullptr;
        if ((e = cudaMalloc(&dm, 8 * (size_t)n)) || (e = cudaMalloc(&vp, 8 * (size_t)n)) || (e = cudaMalloc(&sc, 16)))
            return fail(hs::cuda_error(e, "cudaMalloc (lanczos)"));
        hsm::sqrt_kernel<<<ge, hsm::kThreads, 0, st>>>(n, l1inv, dm);
        hsm::fill_kernel<double><<<ge, hsm::kThreads, 0, st>>>(vv, n, 1.0 / std::sqrt((double)n));
        cudaMemsetAsync(vp, 0, 8 * (size_t)n, st);
        hs::count_launch(2);
        std::vector<double> al, be;
        double beta = 0.0;
        const int rb = hsdev::red_blocks(n);
        for (int j = 0; j < 40 && j < n; ++j) {
            hsm::lanczos_op_kernel<<<gr, hsm::kThreads, 0, st>>>(
                                          n, M64->rp, M64->ci, static_cast<const double*>(M64->v), vv, dm, ww);
            hsdev::dot_partials_kernel<double, double><<<rb, hsdev::kRedThreads, 0, st>>>(ww, vv, n, partials);
            hsdev::finalize_sum_kernel<<<1, hsdev::kRedThreads, 0, st>>>(partials, rb, sc, 0);
            double alpha = 0;
            cudaMemcpyAsync(&alpha, sc, 8, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            hsm::lanczos_update_kernel<<<ge, hsm::kThreads, 0, st>>>(n, ww, vv, vp, alpha, beta);
            hsdev::dot_partials_kernel<double, double><<<rb, hsdev::kRedThreads, 0, st>>>(ww, ww, n, partials);
            hsdev::finalize_sum_kernel<<<1, hsdev::kRedThreads, 0, st>>>(partials, rb, sc, 1);
            double bnext = 0;
            cudaMemcpyAsync(&bnext, sc, 8, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            hs::count_launch(6);
            al.push_back(alpha);
            if (!(bnext > 1e-14 * std::fabs(alpha))) break;
            be.push_back(bnext);
            std::swap(vp, vv);       // v_prev <- v
            hsm::scale_kernel<<<ge, hsm::kThreads, 0, st>>>(n, ww, 1.0 / bnext, vv);
            hs::count_launch();
            beta = bnext;
        }
        be.resize(al.size() > 0 ? al.size() - 1 : 0);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(hs::cuda_error(e, "lanczos"));
        hsm::tridiag_extremes(al, be, S->lmin, S->lmax);
        S->rho = S->lmax;
        cudaFree(dm);
        cudaFree(vp);
        cudaFree(sc);
    }
    if (kind == 1) S->astar = hsm::astar(degree);

    // smoother-precision operands
    if (smoother_dtype == HS_F64) {
        S->A = M64;
        S->l1inv = l1inv;
        l1inv = nullptr;
        M64 = nullptr;
    } else {
        if ((rc = hsm::matrix_from_host(rp, ci, v, HS_F32, st, &S->A))) return fail(rc);
        float* l32 = nullptr;
        if ((e = cudaMalloc(&l32, 4 * (size_t)n))) return fail(hs::cuda_error(e, "cudaMalloc"));
        hsm::convert_kernel<double, float><<<ge, hsm::kThreads, 0, st>>>(l1inv, l32, n);
        hs::count_launch();
        S->l1inv = l32;
    }
    {   // the smoother's matrix in 32-row slices, for its steps
        const int64_t* so = nullptr;
        const int32_t* scl = nullptr;
        const void* sv = nullptr;
        if ((rc = hs::matrix_slices(S->A, st, &so, &scl, &sv))) return fail(rc);
    }
    const size_t es = hsm::dsize(smoother_dtype);
    for (int i = 0; i < 6; ++i)
        if ((e = cudaMalloc(&S->w[i], es * (size_t)n))) return fail(hs::cuda_error(e, "cudaMalloc (work)"));
    if ((e = cudaStreamSynchronize(st))) return fail(hs::cuda_error(e, "chebyshev setup"));
    cudaFree(l1inv);
    cudaFree(vv);
    cudaFree(ww);
    cudaFree(partials);
    cudaFree(rho_d);
    cudaFree(stop);
    hsm::destroy_matrix(M64);
    S->bytes = S->A->bytes + (int64_t)(7 * es * n);
    *out = S;
    return HS_OK;
}

int hs_cheb_smooth(hs_cheb* S, void* x, const void* b, void* stream) {
    if (!S || !x || !b) return hs::set_error(HS_ERR_ARG, "hs_cheb_smooth: NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (S->sdt == HS_F64) return hsm::cheb_smooth_t<double>(S, static_cast<double*>(x), b, HS_F64, false, st);
    return hsm::cheb_smooth_t<float>(S, static_cast<float*>(x), b, HS_F32, false, st);
}

int hs_cheb_apply(hs_cheb* S, const void* r, void* z, int32_t io_dtype, void* stream) {
    if (!S || !r || !z) return hs::set_error(HS_ERR_ARG, "hs_cheb_apply: NULL argument");
    return hs::cheb_apply(S, r, z, io_dtype, static_cast<cudaStream_t>(stream));
}

int hs_cheb_info_get(const hs_cheb* S, hs_cheb_info* info) {
    if (!S || !info) return hs::set_error(HS_ERR_ARG, "hs_cheb_info_get: NULL argument");
    info->n = S->n;
    info->kind = S->kind;
    info->degree = S->degree;
    info->eig = S->eig;
    info->smoother_dtype = S->sdt;
    info->rho = S->rho;
    info->rho_power = S->rho_power;
    info->lanczos_min = S->lmin;
    info->lanczos_max = S->lmax;
    info->astar = S->astar;
    return HS_OK;
}

int hs_cheb_set_rho(hs_cheb* S, double rho) {
    if (!S || !(rho > 0)) return hs::set_error(HS_ERR_ARG, "rho must be positive");
    S->rho = rho;
    return HS_OK;
}

int hs_cheb_destroy(hs_cheb* S) {
    if (S) cudaDeviceSynchronize();
    hsm::destroy_cheb(S);
    return HS_OK;
}

}  // extern "C"

namespace hs {
int cheb_apply(hs_cheb* S, const void* r, void* z, int io, cudaStream_t st) {
    const int32_t n = S->n;
    if (S->sdt == HS_F64) {
        if (io != HS_F64) return set_error(HS_ERR_UNSUPPORTED, "FP64 smoother with FP32 vectors is not provided");
        return hsm::cheb_smooth_t<double>(S, static_cast<double*>(z), r, HS_F64, true, st);
    }
    if (io == HS_F32) return hsm::cheb_smooth_t<float>(S, static_cast<float*>(z), r, HS_F32, true, st);
    // FP64 vectors around an FP32 smoother: r is rounded on the way in, x widened on the way out.
    float* xb = static_cast<float*>(S->w[4]);
    int rc = hsm::cheb_smooth_t<float>(S, xb, r, HS_F64, true, st);
    if (rc) return rc;
    hsm::convert_kernel<float, double><<<hsm::grid_elems(n), hsm::kThreads, 0, st>>>(xb, static_cast<double*>(z), n);
    HS_LAUNCH_CHECK("convert_kernel");
    return HS_OK;
}
}  // namespace hs

// ---------------------------------------------------------------------------
// Chebyshev smoothing without device allocation.
//
// For callers that cannot call cudaMalloc at the point where they smooth: a
// runtime that owns the whole device pool (an XLA/JAX or Julia CUDA.jl
// allocator), code running under an allocator lock, or a serving loop that
// forbids allocation on its hot path.  The caller passes every operand as a
// device buffer it already owns; the smoother's work vectors (r and z, each
// double-buffered) live in one file-scope device array instead of memory from
// cudaMalloc.
//
// The array holds 4 * kNoAllocMaxN doubles (8 MiB) on every GPU that loads
// this library, until the process exits.  All calls on a device share it and
// it keeps the previous call's contents; every element a call reads has been
// written earlier in the same call, so nothing needs clearing.  Calls whose
// GPU work overlaps (two streams, or two host threads) race on the array.
// ---------------------------------------------------------------------------
namespace {
constexpr int32_t kNoAllocMaxN = 262144;
static __device__ __align__(256) double g_cheb_noalloc_scratch[4 * (size_t)kNoAllocMaxN];
double* g_cheb_noalloc_addr[64] = {nullptr};
std::mutex g_cheb_noalloc_mu;
}  // namespace

extern "C" int hs_cheb_smooth_noalloc(int32_t n, int64_t nnz, const int32_t* rp, const int32_t* ci, const double* v,
                                      const double* l1inv, int32_t kind, int32_t degree, double rho, double astar,
                                      double* x, const double* b, void* stream) {
    if (n <= 0 || n > kNoAllocMaxN)
        return hs::set_error(HS_ERR_ARG, "hs_cheb_smooth_noalloc: n = %d outside 1..%d (static scratch limit)", n,
                             kNoAllocMaxN);
    if (nnz < 0 || !rp || !ci || !v || !l1inv || !x || !b)
        return hs::set_error(HS_ERR_ARG, "hs_cheb_smooth_noalloc: NULL operand or negative nnz");
    if (kind != 1 && kind != 4) return hs::set_error(HS_ERR_ARG, "kind must be 1 or 4");
    if (degree < 1) return hs::set_error(HS_ERR_ARG, "degree must be at least 1");
    if (!(rho > 0)) return hs::set_error(HS_ERR_ARG, "rho must be positive");
    if (kind == 1 && !(astar > 0 && astar < 1)) return hs::set_error(HS_ERR_ARG, "astar must lie in (0, 1)");
    int dev = 0;
    HS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return hs::set_error(HS_ERR_ARG, "device index out of range");
    double* scratch = nullptr;
    {
        // First call on this device (the device current here): resolve the
        // device address of the array.  The host-side symbol is only a
        // stand-in, never a device pointer.
        std::lock_guard<std::mutex> lk(g_cheb_noalloc_mu);
        if (!g_cheb_noalloc_addr[dev]) {
            void* p = nullptr;
            HS_CUDA(cudaGetSymbolAddress(&p, g_cheb_noalloc_scratch));
            g_cheb_noalloc_addr[dev] = static_cast<double*>(p);
        }
        scratch = g_cheb_noalloc_addr[dev];
    }
    hs_matrix M;
    M.n = n;
    M.nnz = nnz;
    M.dtype = HS_F64;
    M.rp = const_cast<int32_t*>(rp);
    M.ci = const_cast<int32_t*>(ci);
    M.v = const_cast<double*>(v);
    hs_cheb S;
    S.n = n;
    S.kind = kind;
    S.degree = degree;
    S.sdt = HS_F64;
    S.rho = rho;
    S.astar = kind == 1 ? astar : 0.0;
    S.A = &M;
    S.l1inv = const_cast<double*>(l1inv);
    for (int i = 0; i < 4; ++i) S.w[i] = scratch + (size_t)i * n;
    const int rc = hsm::cheb_smooth_t<double>(&S, x, b, HS_F64, false, static_cast<cudaStream_t>(stream));
    S.A = nullptr;      // stack descriptors own nothing
    S.l1inv = nullptr;
    for (int i = 0; i < 4; ++i) S.w[i] = nullptr;
    return rc;
}

namespace hsdev {

__global__ void slice_width_kernel(int32_t n, int64_t nslices, const int32_t* __restrict__ rp,
                                   int64_t* __restrict__ ent) {
    const int lane = threadIdx.x & 31;
    for (int64_t sl = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; sl <= nslices;
         sl += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t row = sl * 32 + lane;
        const int32_t len = (sl < nslices && row < n) ? rp[row + 1] - rp[row] : 0;
        const int32_t w = (int32_t)__reduce_max_sync(0xffffffffu, (unsigned)len);
        if (lane == 0) ent[sl] = 32 * (int64_t)w;
    }
}

}  // namespace hsdev
