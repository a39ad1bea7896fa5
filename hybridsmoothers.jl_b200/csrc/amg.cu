// The L1GS preconditioner as an algebraic-multigrid smoother.
//
// Reference: ext/HybridSmoothersAMGExt.jl (HybridSmoothers.jl v0.1.4).  The
// extension wraps a preconditioner P and the level matrix A in a
// HybridSmoother (:8-13) whose smooth! (:26-33) runs two Richardson sweeps
//   mul!(residual, A, x); residual .-= b; ldiv!(correction, P, residual);
//   x .-= correction
// Here one sweep is two launches: a warp CSR-stream kernel that forms
// residual_i = (A x)_i - b_i (the row sum in storage order from zero, then one
// rounded subtraction, as the three-argument mul! and the broadcast do), and
// the L1GS apply.  From the second sweep on, the residual kernel also applies
// the previous correction: the x it multiplies is x_j - correction_j,
// recomputed per use with the same single subtraction, and it stores the
// updated x of its own rows into a separate buffer (x is never written while
// other blocks read it).  The last correction is applied by an element-wise
// kernel into the caller's x.  Every value is bitwise the reference's
// sequence.
#include <algorithm>

#include "internal.cuh"
#include "spmv.cuh"

struct hs_richardson_s {
    const hs_matrix* A = nullptr;
    hs_l1gs* P = nullptr;
    int32_t n = 0, dtype = HS_F64;
    void* residual = nullptr;
    void* correction = nullptr;
    void* xbuf[2] = {nullptr, nullptr};
    const int64_t* soff = nullptr;   // the matrix's 32-row slices (owned by the matrix)
    const int32_t* scol = nullptr;
    const void* sval = nullptr;
};

namespace {

// residual = A xin - b, where xin_j = x_j (first sweep) or x_j - z_j (later
// sweeps, also stored into xout for the rows of this warp).  Over the matrix's
// 32-row slices (spmv.cuh) when soff is given, else warp CSR-stream: the same
// fold either way.
constexpr int kRT = 256;

template <typename T, bool UPDATE>
__global__ void __launch_bounds__(kRT)
    richardson_residual(int32_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                        const T* __restrict__ v, const int64_t* __restrict__ soff, const int32_t* __restrict__ scol,
                        const T* __restrict__ sval, const T* __restrict__ x, const T* __restrict__ z,
                        const T* __restrict__ b, T* __restrict__ r, T* __restrict__ xout) {
    __shared__ T wbuf[kRT / 32][hsdev::kWarpCap];
    const int warp = threadIdx.x >> 5;
    auto xin = [&](int32_t j) {
        if (UPDATE) return sub_rn(__ldg(x + j), __ldg(z + j));
        return __ldg(x + j);
    };
    for (int64_t row0 = ((int64_t)blockIdx.x * (kRT / 32) + warp) * 32; row0 < n; row0 += (int64_t)gridDim.x * kRT) {
        const T acc = soff ? hsdev::slice_row_fold(soff[row0 >> 5], soff[(row0 >> 5) + 1], scol, sval, T(0), xin,
                                                   hsdev::AddOp<T>())
                           : hsdev::csr_warp_fold(wbuf[warp], n, rp, ci, v, row0, T(0), xin, hsdev::AddOp<T>());
        const int64_t i = row0 + (threadIdx.x & 31);
        if (i < n) {
            r[i] = sub_rn(acc, b[i]);
            if (UPDATE) xout[i] = xin((int32_t)i);
        }
    }
}

template <typename T>
__global__ void richardson_finish(int32_t n, const T* __restrict__ xin, const T* __restrict__ z, T* __restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = sub_rn(xin[i], z[i]);
}

template <typename T>
int smooth_t(hs_richardson* S, T* x, const T* b, int sweeps, cudaStream_t st) {
    const int32_t n = S->n;
    const int32_t *rp = nullptr, *ci = nullptr;
    const void* vv = nullptr;
    int dt = 0;
    hs::matrix_arrays(S->A, &rp, &ci, &vv, &dt);
    const T* v = static_cast<const T*>(vv);
    const int64_t* so = S->soff;
    const int32_t* sc = S->scol;
    const T* sv = static_cast<const T*>(S->sval);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + kRT - 1) / kRT, INT32_MAX));
    T* r = static_cast<T*>(S->residual);
    T* z = static_cast<T*>(S->correction);
    const T* xcur = x;
    int nb = 0;
    int rc;
    for (int k = 0; k < sweeps; ++k) {
        T* xnext = static_cast<T*>(S->xbuf[nb]);
        if (k == 0) {
            richardson_residual<T, false><<<grid, kRT, 0, st>>>(n, rp, ci, v, so, sc, sv, xcur, z, b, r, nullptr);
        } else {
            richardson_residual<T, true><<<grid, kRT, 0, st>>>(n, rp, ci, v, so, sc, sv, xcur, z, b, r, xnext);
            xcur = xnext;
            nb ^= 1;
        }
        HS_LAUNCH_CHECK("richardson_residual");
        if ((rc = hs_l1gs_apply(S->P, r, z, S->dtype, st))) return rc;
    }
    const int ge = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)hs::num_sms() * 16));
    richardson_finish<T><<<ge, 256, 0, st>>>(n, xcur, z, x);
    HS_LAUNCH_CHECK("richardson_finish");
    return HS_OK;
}

}  // namespace

extern "C" {

int hs_richardson_create(const hs_matrix* A, hs_l1gs* P, hs_richardson** out) {
    if (!A || !P || !out) return hs::set_error(HS_ERR_ARG, "hs_richardson_create: NULL argument");
    *out = nullptr;
    hs_l1gs_info pi;
    int rc = hs_l1gs_info_get(P, &pi);
    if (rc) return rc;
    const int32_t n = hs::matrix_n(A);
    const int32_t *rp, *ci;
    const void* v;
    int dt = 0;
    hs::matrix_arrays(A, &rp, &ci, &v, &dt);
    if (pi.n != n) return hs::set_error(HS_ERR_ARG, "preconditioner size %d != matrix size %d", pi.n, n);
    if (pi.smoother_dtype == HS_F64 && dt == HS_F32)
        return hs::set_error(HS_ERR_UNSUPPORTED, "an FP64 smoother with an FP32 matrix is not provided");
    hs_richardson* S = new hs_richardson_s();
    S->A = A;
    S->P = P;
    S->n = n;
    S->dtype = dt;
    // the matrix in 32-row slices (kept with the matrix; built once)
    if ((rc = hs::matrix_slices(const_cast<hs_matrix*>(A), nullptr, &S->soff, &S->scol, &S->sval))) {
        delete S;
        return rc;
    }
    const size_t bytes = (dt == HS_F64 ? 8 : 4) * (size_t)n;
    cudaError_t e;
    if ((e = cudaMalloc(&S->residual, bytes)) || (e = cudaMalloc(&S->correction, bytes)) ||
        (e = cudaMalloc(&S->xbuf[0], bytes)) || (e = cudaMalloc(&S->xbuf[1], bytes))) {
        hs_richardson_destroy(S);
        return hs::cuda_error(e, "cudaMalloc (richardson smoother)");
    }
    *out = S;
    return HS_OK;
}

int hs_richardson_smooth(hs_richardson* S, void* x, const void* b, int32_t sweeps, void* stream) {
    if (!S || !x || !b) return hs::set_error(HS_ERR_ARG, "hs_richardson_smooth: NULL argument");
    if (sweeps < 1) return hs::set_error(HS_ERR_ARG, "sweeps must be positive");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (S->dtype == HS_F64)
        return smooth_t<double>(S, static_cast<double*>(x), static_cast<const double*>(b), sweeps, st);
    return smooth_t<float>(S, static_cast<float*>(x), static_cast<const float*>(b), sweeps, st);
}

int hs_richardson_destroy(hs_richardson* S) {
    if (!S) return HS_OK;
    cudaDeviceSynchronize();
    cudaFree(S->residual);
    cudaFree(S->correction);
    cudaFree(S->xbuf[0]);
    cudaFree(S->xbuf[1]);
    delete S;
    return HS_OK;
}

}  // extern "C"
