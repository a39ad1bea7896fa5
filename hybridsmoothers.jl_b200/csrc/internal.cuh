// Cross-file internal interfaces of libhsb200 (not part of the C ABI).
#pragma once

#include "hs_common.cuh"

namespace hs {

int matrix_spmv(const hs_matrix* M, const void* x, void* y, double alpha, double beta, cudaStream_t st);
int matrix_n(const hs_matrix* M);
int64_t matrix_nnz(const hs_matrix* M);
void matrix_arrays(const hs_matrix* M, const int32_t** rp, const int32_t** ci, const void** v, int* dtype);
// The matrix in 32-row slices (spmv.cuh; values in the matrix type), built
// at the first call and kept with the matrix.
int matrix_slices(hs_matrix* M, cudaStream_t st, const int64_t** soff, const int32_t** scol, const void** sval);
int cheb_apply(hs_cheb* S, const void* r, void* z, int io, cudaStream_t st);
// Uploads a validated host matrix as device CSR in `dtype` (a CSC input is
// transposed on the device); rp has n+1 entries, ci and v nnz.  For a CSC
// input, a non-null `diag` (n entries) receives DiagonalIndices and *bad
// (initialised by the caller to n) the smallest column whose diagonal is
// missing or zero.
// The device's default stream-ordered pool keeps what it has reserved.
void keep_pool_reserve();
int csr_from_host(const hs_sparse* A, int32_t dtype, int32_t* rp, int32_t* ci, void* v, cudaStream_t st,
                  int32_t* diag = nullptr, int32_t* bad = nullptr);

// The device-side pieces of an L1GS preconditioner that a batched launch needs.
struct L1gsView {
    int32_t n, ps, ngroups, tlen;
    int64_t npad;
    const void* Di;
    const void* SLi;
    const void* SUi;
    int32_t sdt, sweep, cache;
};
int l1gs_view_of(const hs_l1gs* P, L1gsView* v);
// Symmetric packed-cache L1GS built from a device CSR matrix (read during the
// call only; for a symmetric matrix its rows are the CSC columns isSymA reads).
int l1gs_create_from_matrix(const hs_matrix* M, int32_t partsize, double eta, int32_t sweep, int32_t smoother_dtype,
                            cudaStream_t st, hs_l1gs** out);
// Its buffers are stream-ordered: free them in order on `st` (no device sync).
void l1gs_destroy_async(hs_l1gs* P, cudaStream_t st);
// Device CSR matrix with stream-ordered buffers (allocated on `st`).
int matrix_create_async(const hs_sparse* A, int32_t dtype, cudaStream_t st, hs_matrix** out);
void matrix_destroy_async(hs_matrix* M, cudaStream_t st);

}  // namespace hs
