// Cross-file internal interfaces of libhsb200 (not part of the C ABI).
#pragma once

#include "hs_common.cuh"

namespace hs {

int matrix_spmv(const hs_matrix* M, const void* x, void* y, double alpha, double beta, cudaStream_t st);
int matrix_n(const hs_matrix* M);
void matrix_arrays(const hs_matrix* M, const int32_t** rp, const int32_t** ci, const void** v, int* dtype);
int cheb_apply(hs_cheb* S, const void* r, void* z, int io, cudaStream_t st);

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

}  // namespace hs
