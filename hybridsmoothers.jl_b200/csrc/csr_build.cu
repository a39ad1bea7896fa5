// Device-side CSR construction for hs_matrix_create.
//
// SparseMatricesCSR.jl's mul! reads a row-wise matrix; a SparseMatrixCSC
// input is first turned into CSR (the reference's adapt step then moves the
// CSR to the device).  Doing that transpose on the host costs a scattered
// O(nnz) pass per matrix; here the CSC arrays are uploaded as they are and
// transposed on the GPU: the row index of every entry is the key of a stable
// radix sort whose payload is the entry's storage position, so the entries of
// each row come out in ascending column order (CSC enumerates columns in
// order) -- exactly the host transpose's output.
#include <algorithm>
#include <mutex>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "internal.cuh"

namespace {

__global__ void expand_columns(int32_t n, const int32_t* __restrict__ ptr, int32_t* __restrict__ col) {
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        for (int32_t q = ptr[c]; q < ptr[c + 1]; ++q) col[q] = c;
}

__global__ void iota_kernel(int64_t m, int32_t* __restrict__ a) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = (int32_t)i;
}

// rp[r] = first sorted position whose row is >= r.  Thread k owns the rows in
// (row[k-1], row[k]], with row[-1] = -1 and row[nnz] = n.
__global__ void row_pointers(int32_t n, int64_t nnz, const int32_t* __restrict__ rows, int32_t* __restrict__ rp) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t prev = k == 0 ? -1 : rows[k - 1];
        const int32_t cur = k == nnz ? n : rows[k];
        for (int32_t r = prev + 1; r <= cur; ++r) rp[r] = (int32_t)k;
    }
}

template <typename TS, typename TD>
__global__ void gather_entries(int64_t nnz, const int32_t* __restrict__ perm, const int32_t* __restrict__ col,
                               const TS* __restrict__ val, int32_t* __restrict__ ci, TD* __restrict__ v) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t q = perm[k];
        ci[k] = col[q];
        v[k] = (TD)val[q];
    }
}

template <typename TS, typename TD>
__global__ void convert_values(int64_t m, const TS* __restrict__ a, TD* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (TD)a[i];
}

// DiagonalIndices (src/l1_gauss_seidel.jl:422-436) on the uploaded CSC:
// diag[c] = position of A[c,c] in rowval (binary search of the sorted
// column); a missing or zero diagonal records its column in *bad
// (atomicMin: the smallest such column, the one the reference's ascending
// loop throws SingularException for).
template <typename TS>
__global__ void diag_indices_kernel(int32_t n, const int32_t* __restrict__ ptr, const int32_t* __restrict__ rows,
                                    const TS* __restrict__ val, int32_t* __restrict__ diag, int32_t* __restrict__ bad) {
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int32_t lo = ptr[c], hi = ptr[c + 1];   // first position with rows[pos] >= c in [lo, hi)
        while (lo < hi) {
            const int32_t mid = lo + (hi - lo) / 2;
            if (rows[mid] < c) lo = mid + 1;
            else hi = mid;
        }
        const bool ok = lo < ptr[c + 1] && rows[lo] == c && val[lo] != TS(0);
        diag[c] = ok ? lo : -1;
        if (!ok) atomicMin(bad, c);
    }
}

int grid_for(int64_t m) { return (int)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, 8192)); }

template <typename TS, typename TD>
int gather_t(int64_t nnz, const int32_t* perm, const int32_t* col, const void* val, int32_t* ci, void* v,
             cudaStream_t st) {
    gather_entries<TS, TD><<<grid_for(nnz), 256, 0, st>>>(nnz, perm, col, static_cast<const TS*>(val), ci,
                                                          static_cast<TD*>(v));
    HS_LAUNCH_CHECK("gather_entries");
    return HS_OK;
}

template <typename TS, typename TD>
int convert_t(int64_t m, const void* a, void* b, cudaStream_t st) {
    convert_values<TS, TD><<<grid_for(m), 256, 0, st>>>(m, static_cast<const TS*>(a), static_cast<TD*>(b));
    HS_LAUNCH_CHECK("convert_values");
    return HS_OK;
}

// Temporaries in stream order: freed on the stream after the work that uses them.
struct AsyncBufs {
    cudaStream_t st;
    std::vector<void*> p;
    ~AsyncBufs() {
        for (void* q : p) cudaFreeAsync(q, st);
    }
    int get(void** out, size_t bytes) {
        cudaError_t e = cudaMallocAsync(out, bytes ? bytes : 8, st);
        if (e != cudaSuccess) return hs::cuda_error(e, "cudaMallocAsync (CSR build)");
        p.push_back(*out);
        return HS_OK;
    }
};

}  // namespace

namespace hs {

// The temporaries come from the device's default stream-ordered pool; keep
// what it has reserved between calls (a served stream builds one matrix per
// request) instead of returning it to the driver at every synchronisation.
void keep_pool_reserve() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done[dev] = true;
}

int csr_from_host(const hs_sparse* A, int32_t dtype, int32_t* rp, int32_t* ci, void* v, cudaStream_t st,
                  int32_t* diag, int32_t* bad) {
    keep_pool_reserve();
    const int32_t n = A->n;
    const int64_t nnz = A->nnz;
    const size_t ses = A->dtype == HS_F64 ? 8 : 4;
    AsyncBufs tmp{st, {}};
    int rc;
    if (A->format == HS_CSR) {
        HS_CUDA(cudaMemcpyAsync(rp, A->ptr, sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, st));
        if (nnz == 0) return HS_OK;
        HS_CUDA(cudaMemcpyAsync(ci, A->idx, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
        if (A->dtype == dtype) {
            HS_CUDA(cudaMemcpyAsync(v, A->val, ses * nnz, cudaMemcpyHostToDevice, st));
            return HS_OK;
        }
        void* raw = nullptr;
        if ((rc = tmp.get(&raw, ses * nnz))) return rc;
        HS_CUDA(cudaMemcpyAsync(raw, A->val, ses * nnz, cudaMemcpyHostToDevice, st));
        return A->dtype == HS_F64 ? convert_t<double, float>(nnz, raw, v, st)
                                  : convert_t<float, double>(nnz, raw, v, st);
    }
    // CSC: upload, expand column indices, stable sort by row, gather.
    void *ptr = nullptr, *rows_in = nullptr, *rows_out = nullptr, *col = nullptr, *pos = nullptr, *perm = nullptr,
         *val = nullptr;
    if ((rc = tmp.get(&ptr, sizeof(int32_t) * (n + 1))) || (rc = tmp.get(&rows_in, sizeof(int32_t) * nnz)) ||
        (rc = tmp.get(&rows_out, sizeof(int32_t) * nnz)) || (rc = tmp.get(&col, sizeof(int32_t) * nnz)) ||
        (rc = tmp.get(&pos, sizeof(int32_t) * nnz)) || (rc = tmp.get(&perm, sizeof(int32_t) * nnz)) ||
        (rc = tmp.get(&val, ses * nnz)))
        return rc;
    HS_CUDA(cudaMemcpyAsync(ptr, A->ptr, sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, st));
    if (nnz > 0) {
        HS_CUDA(cudaMemcpyAsync(rows_in, A->idx, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
        HS_CUDA(cudaMemcpyAsync(val, A->val, ses * nnz, cudaMemcpyHostToDevice, st));
    }
    if (diag) {
        if (A->dtype == HS_F64)
            diag_indices_kernel<double><<<grid_for(n), 256, 0, st>>>(n, static_cast<const int32_t*>(ptr),
                                                                     static_cast<const int32_t*>(rows_in),
                                                                     static_cast<const double*>(val), diag, bad);
        else
            diag_indices_kernel<float><<<grid_for(n), 256, 0, st>>>(n, static_cast<const int32_t*>(ptr),
                                                                    static_cast<const int32_t*>(rows_in),
                                                                    static_cast<const float*>(val), diag, bad);
        HS_LAUNCH_CHECK("diag_indices_kernel");
    }
    expand_columns<<<grid_for(n), 256, 0, st>>>(n, static_cast<const int32_t*>(ptr), static_cast<int32_t*>(col));
    iota_kernel<<<grid_for(nnz), 256, 0, st>>>(nnz, static_cast<int32_t*>(pos));
    hs::count_launch();
    HS_LAUNCH_CHECK("expand_columns");
    int end_bit = 1;
    while (end_bit < 31 && ((int64_t)1 << end_bit) < (int64_t)n) ++end_bit;
    if (nnz > 0) {
        size_t tbytes = 0;
        const int32_t *ki = static_cast<const int32_t*>(rows_in), *vi = static_cast<const int32_t*>(pos);
        int32_t *ko = static_cast<int32_t*>(rows_out), *vo = static_cast<int32_t*>(perm);
        HS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tbytes, ki, ko, vi, vo, nnz, 0, end_bit, st));
        void* ttmp = nullptr;
        if ((rc = tmp.get(&ttmp, tbytes))) return rc;
        HS_CUDA(cub::DeviceRadixSort::SortPairs(ttmp, tbytes, ki, ko, vi, vo, nnz, 0, end_bit, st));
    }
    row_pointers<<<grid_for(nnz + 1), 256, 0, st>>>(n, nnz, static_cast<const int32_t*>(rows_out), rp);
    HS_LAUNCH_CHECK("row_pointers");
    if (nnz == 0) return HS_OK;
    const int32_t* pm = static_cast<const int32_t*>(perm);
    const int32_t* cl = static_cast<const int32_t*>(col);
    if (A->dtype == HS_F64)
        return dtype == HS_F64 ? gather_t<double, double>(nnz, pm, cl, val, ci, v, st)
                               : gather_t<double, float>(nnz, pm, cl, val, ci, v, st);
    return dtype == HS_F64 ? gather_t<float, double>(nnz, pm, cl, val, ci, v, st)
                           : gather_t<float, float>(nnz, pm, cl, val, ci, v, st);
}

}  // namespace hs
