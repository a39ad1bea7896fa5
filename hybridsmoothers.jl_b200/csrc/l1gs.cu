// L1 Gauss-Seidel preconditioner for B200 (sm_100a): setup and apply.
//
// Reference: src/l1_gauss_seidel.jl of HybridSmoothers.jl v0.1.4.
//
// Storage (packed cache).  The reference keeps each partition's strict
// triangle row-major in its own block (:480-502) and walks it with one thread
// per partition, so neighbouring threads read addresses ps(ps-1)/2 elements
// apart.  Here the same values live in an interleaved ("partition-minor")
// layout: element e of partition k sits at e*npad + k, with npad = nparts
// rounded up to a multiple of 32.  A warp owns 32 consecutive partitions, one
// per lane, and every stream element of the warp is one contiguous 128/256-byte
// row, fetched as a [E x 32] tile by a 2D TMA load into a per-warp ring of
// shared-memory stages.  Element order inside a partition is the order the
// sweep consumes it:
//   lower stream  e = li(li-1)/2 + lj                      (rows ascending)
//   upper stream  e = q(q-1)/2 + (lj-li-1), q = ps-1-li    (rows descending)
// D_Dl1 is kept in natural order (D) and, for the packed kernels, also
// interleaved as Di[li*npad + k].  Introspection (hs_l1gs_get_packed)
// converts back to the reference layout.
//
// Arithmetic.  Each row accumulates acc = sum_j a_ij*y_j in ascending j with
// separately rounded multiply and add, then y_i = (y_i - acc) / D_i, exactly
// the reference's sequence (:1090-1092, :1547-1585), so results are bitwise
// equal to the reference order of operations.
#include <algorithm>
#include <cstring>
#include <vector>

#include "hs_common.cuh"

namespace {

constexpr int kWarpsPerBlock = 4;

__host__ __device__ __forceinline__ int64_t lo_idx(int64_t li, int64_t lj) { return li * (li - 1) / 2 + lj; }
__host__ __device__ __forceinline__ int64_t up_idx(int64_t ps, int64_t li, int64_t lj) {
    int64_t q = ps - 1 - li;
    return q * (q - 1) / 2 + (lj - li - 1);
}

// ---------------------------------------------------------------------------
// Setup: D_Dl1 and packing, one thread per row.
//   D_Dl1: _diag_offpart_rowwise (:1101-1129) + eta rule (:1017-1022)
//   packing: _pack_strict_lower/upper_rowwise! (:1248-1277, :1380-1413)
// TM is the matrix value type (the type D_Dl1 is computed in), TS the
// smoother type it is stored in.
// ---------------------------------------------------------------------------
template <typename TM, typename TS>
__global__ void setup_rows_kernel(int32_t n, int32_t ps, int64_t npad, const int32_t* __restrict__ rp,
                                  const int32_t* __restrict__ ci, const TM* __restrict__ v, TM eta,
                                  TS* __restrict__ D, TS* __restrict__ Di, TS* __restrict__ SLi,
                                  TS* __restrict__ SUi) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t k = i / ps;
    const int64_t s = k * ps;
    const int64_t e = min(s + ps - 1, (int64_t)n - 1);
    const int64_t li = i - s;
    TM b = TM(0), d = TM(0);
    for (int32_t p = rp[i]; p < rp[i + 1]; ++p) {
        const int64_t j = ci[p];
        const TM val = v[p];
        if (j == i) {
            b = val;
        } else if (j < s || j > e) {
            d = add_rn(d, abs_t(val));
        } else if (j < i) {
            if (SLi) SLi[lo_idx(li, j - s) * npad + k] = (TS)val;
        } else {
            if (SUi) SUi[up_idx(ps, li, j - s) * npad + k] = (TS)val;
        }
    }
    const TM dl1star = (b >= mul_rn(eta, d)) ? TM(0) : div_rn(d, TM(2));
    const TM Dv = add_rn(b, dl1star);
    D[i] = (TS)Dv;
    if (Di) Di[li * npad + k] = (TS)Dv;
}

template <typename T>
__global__ void fill_kernel(T* p, int64_t count, T value) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = value;
}

template <typename TA, typename TB>
__global__ void convert_kernel(const TA* __restrict__ a, TB* __restrict__ b, int64_t count) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (TB)a[i];
}

// ---------------------------------------------------------------------------
// Packed apply: thread per partition, warp per 32 partitions, TMA ring.
// ---------------------------------------------------------------------------
struct PackedParams {
    int32_t n, ps, nparts;
    int64_t npad;
    int32_t ngroups;
    int64_t tlen;      // ps(ps-1)/2 stream elements per direction
    int32_t ntiles;    // ceil(tlen / E) tiles per direction
    const void* Di;
    const void* x;
    void* y;
    int32_t* err;
    int32_t ys_stride; // 33
    uint32_t warp_bytes;
    uint32_t ring_bytes;
};

// Issue tile c of this warp's tile sequence.
template <typename T, int E, int STAGES, int SWEEP>
__device__ __forceinline__ void issue_tile(const CUtensorMap* tmL, const CUtensorMap* tmU, T* buf, uint64_t* bars,
                                           int64_t c, int32_t g0, int32_t gstride, int32_t ntiles) {
    const int32_t ntpg = (SWEEP == 2) ? 2 * ntiles : ntiles;
    const int64_t gi = c / ntpg;
    int32_t ti = (int32_t)(c - gi * ntpg);
    const int32_t g = g0 + (int32_t)gi * gstride;
    const CUtensorMap* map = (SWEEP == 1) ? tmU : tmL;
    if (SWEEP == 2 && ti >= ntiles) {
        map = tmU;
        ti -= ntiles;
    }
    const int stage = (int)(c % STAGES);
    uint64_t* bar = bars + stage;
    hsdev::mbar_arrive_expect_tx(bar, (uint32_t)(E * 32 * sizeof(T)));
    hsdev::tma_load_2d(buf + (size_t)stage * E * 32, map, g * 32, ti * E, bar);
}

template <typename T, typename IO, int SWEEP, int E, int STAGES>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    l1gs_packed_kernel(const __grid_constant__ CUtensorMap tmL, const __grid_constant__ CUtensorMap tmU,
                       const PackedParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    unsigned char* wbase = smem + (size_t)warp * p.warp_bytes;
    T* ring = reinterpret_cast<T*>(wbase);
    uint64_t* bars = reinterpret_cast<uint64_t*>(wbase + p.ring_bytes);
    T* ys = reinterpret_cast<T*>(wbase + p.ring_bytes + 8 * STAGES);
    const int S = p.ys_stride;
    const T* __restrict__ Di = static_cast<const T*>(p.Di);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);

    const int wpb = blockDim.x >> 5;
    const int32_t g0 = blockIdx.x * wpb + warp;
    const int32_t gstride = gridDim.x * wpb;
    const int64_t my_groups = g0 < p.ngroups ? (int64_t)(p.ngroups - 1 - g0) / gstride + 1 : 0;
    const int32_t ntpg = (SWEEP == 2) ? 2 * p.ntiles : p.ntiles;
    const int64_t total = my_groups * ntpg;

    if (lane == 0) {
        if (total > 0) {
            hsdev::prefetch_tensormap(&tmL);
            if (SWEEP != 0) hsdev::prefetch_tensormap(&tmU);
        }
        for (int s = 0; s < STAGES; ++s) hsdev::mbar_init(bars + s, 1);
        hsdev::fence_barrier_init();
        const int64_t pro = total < STAGES ? total : STAGES;
        for (int64_t c = 0; c < pro; ++c)
            issue_tile<T, E, STAGES, SWEEP>(&tmL, &tmU, ring, bars, c, g0, gstride, p.ntiles);
    }
    __syncwarp();

    int64_t c = 0;       // tile being consumed
    int32_t r = 0;       // row inside it
    const T* cur = nullptr;
    bool abort = false;

    // Wait for tile c; false if the bounded wait ran out on any lane.
    auto wait_tile = [&]() -> bool {
        const int stage = (int)(c % STAGES);
        const uint32_t parity = (uint32_t)((c / STAGES) & 1);
        const bool ok = hsdev::mbar_wait_bounded(bars + stage, parity);
        cur = ring + (size_t)stage * E * 32;
        return __all_sync(0xffffffffu, ok);
    };
    // All lanes are done with tile c: refill its stage with tile c+STAGES.
    auto finish_tile = [&]() {
        __syncwarp();
        if (lane == 0) {
            hsdev::fence_proxy_async_smem();
            if (c + STAGES < total)
                issue_tile<T, E, STAGES, SWEEP>(&tmL, &tmU, ring, bars, c + STAGES, g0, gstride, p.ntiles);
        }
        ++c;
        r = 0;
    };

    const int ps = p.ps;
    for (int64_t gi = 0; gi < my_groups && !abort; ++gi) {
        const int64_t g = g0 + gi * gstride;
        const int64_t k = g * 32 + lane;
        const int64_t rowbase = g * 32 * (int64_t)ps;
        // x -> ys (transpose through shared memory, coalesced global reads)
        for (int t = lane; t < 32 * ps; t += 32) {
            const int64_t row = rowbase + t;
            const T v = row < p.n ? (T)x[row] : T(0);
            ys[(t % ps) * S + t / ps] = v;
        }
        __syncwarp();

        if (SWEEP != 1) {  // forward, lower stream
            for (int li = 0; li < ps && !abort; ++li) {
                T acc = T(0);
                for (int lj = 0; lj < li; ++lj) {
                    if (r == 0) {
                        if (!wait_tile()) { abort = true; break; }
                    }
                    acc = add_rn(acc, mul_rn(cur[r * 32 + lane], ys[lj * S + lane]));
                    if (++r == E) finish_tile();
                }
                if (abort) break;
                const T d = Di[(int64_t)li * p.npad + k];
                ys[li * S + lane] = div_rn(sub_rn(ys[li * S + lane], acc), d);
            }
            if (!abort && r != 0) finish_tile();
        }
        if (SWEEP == 2 && !abort) {  // y .= D_Dl1 .* y  (:897)
            for (int li = 0; li < ps; ++li)
                ys[li * S + lane] = mul_rn(Di[(int64_t)li * p.npad + k], ys[li * S + lane]);
        }
        if (SWEEP != 0 && !abort) {  // backward, upper stream
            for (int li = ps - 1; li >= 0 && !abort; --li) {
                T acc = T(0);
                for (int lj = li + 1; lj < ps; ++lj) {
                    if (r == 0) {
                        if (!wait_tile()) { abort = true; break; }
                    }
                    acc = add_rn(acc, mul_rn(cur[r * 32 + lane], ys[lj * S + lane]));
                    if (++r == E) finish_tile();
                }
                if (abort) break;
                const T d = Di[(int64_t)li * p.npad + k];
                ys[li * S + lane] = div_rn(sub_rn(ys[li * S + lane], acc), d);
            }
            if (!abort && r != 0) finish_tile();
        }
        if (abort) break;
        __syncwarp();
        for (int t = lane; t < 32 * ps; t += 32) {
            const int64_t row = rowbase + t;
            if (row < p.n) y[row] = (IO)ys[(t % ps) * S + t / ps];
        }
        __syncwarp();
    }

    if (abort) {
        // Record the timeout, then let every copy already in flight land
        // (bounded) before the CTA's shared memory goes away.
        if (lane == 0) hsdev::report_error(p.err, hsdev::kErrWaitTimeout);
        const int64_t issued_end = (c + STAGES < total) ? c + STAGES : total;
        for (int64_t cc = c; cc < issued_end; ++cc)
            (void)hsdev::mbar_wait_bounded(bars + (int)(cc % STAGES), (uint32_t)((cc / STAGES) & 1));
    }
}

// ---------------------------------------------------------------------------
// View apply (MatrixViewCache): warp per partition.  The warp gathers the
// partition's in-block strict-lower and strict-upper entries from the row-wise
// matrix into shared memory (ascending column per row, like the reference's
// row scan :1588-1597, :1700-1709), then lane 0 runs the serial row recurrence.
// A partition whose in-block entries exceed the shared capacity is solved by
// scanning its rows in global memory instead (same arithmetic).
// ---------------------------------------------------------------------------
struct ViewParams {
    int32_t n, ps, nparts;
    const int32_t* rp;
    const int32_t* ci;
    const void* v;
    const void* D;
    const void* x;
    void* y;
    int32_t cap_lo, cap_up;
    uint32_t warp_bytes;
};

template <typename T, typename IO, int SWEEP>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) l1gs_view_kernel(const ViewParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int ps = p.ps;
    unsigned char* w = smem + (size_t)warp * p.warp_bytes;
    T* ys = reinterpret_cast<T*>(w);
    T* ds = ys + ps;
    T* lo_val = ds + ps;
    T* up_val = lo_val + p.cap_lo;
    int32_t* lo_off = reinterpret_cast<int32_t*>(up_val + p.cap_up);
    int32_t* up_off = lo_off + ps + 1;
    uint16_t* lo_col = reinterpret_cast<uint16_t*>(up_off + ps + 1);
    uint16_t* up_col = lo_col + p.cap_lo;

    const int32_t* __restrict__ rp = p.rp;
    const int32_t* __restrict__ ci = p.ci;
    const T* __restrict__ v = static_cast<const T*>(p.v);
    const T* __restrict__ D = static_cast<const T*>(p.D);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);
    const bool want_lo = SWEEP != 1, want_up = SWEEP != 0;

    const int wpb = blockDim.x >> 5;
    for (int64_t k = (int64_t)blockIdx.x * wpb + warp; k < p.nparts; k += (int64_t)gridDim.x * wpb) {
        const int64_t s = k * ps;
        const int64_t e = min(s + ps - 1, (int64_t)p.n - 1);
        const int aps = (int)(e - s + 1);
        int carry_lo = 0, carry_up = 0;
        for (int base = 0; base < aps; base += 32) {
            const int li = base + lane;
            const bool valid = li < aps;
            const int64_t i = s + li;
            int cl = 0, cu = 0, p0 = 0, p1 = 0;
            if (valid) {
                ys[li] = (T)x[i];
                ds[li] = D[i];
                p0 = rp[i];
                p1 = rp[i + 1];
                for (int q = p0; q < p1; ++q) {
                    const int64_t j = ci[q];
                    cl += (want_lo && j >= s && j < i);
                    cu += (want_up && j > i && j <= e);
                }
            }
            // exclusive warp scans
            int il = cl, iu = cu;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int tl = __shfl_up_sync(0xffffffffu, il, o);
                const int tu = __shfl_up_sync(0xffffffffu, iu, o);
                if (lane >= o) { il += tl; iu += tu; }
            }
            const int ol = carry_lo + il - cl, ou = carry_up + iu - cu;
            if (valid) {
                lo_off[li] = ol;
                up_off[li] = ou;
                int wl = ol, wu = ou;
                for (int q = p0; q < p1; ++q) {
                    const int64_t j = ci[q];
                    if (want_lo && j >= s && j < i) {
                        if (wl < p.cap_lo) { lo_col[wl] = (uint16_t)(j - s); lo_val[wl] = v[q]; }
                        ++wl;
                    } else if (want_up && j > i && j <= e) {
                        if (wu < p.cap_up) { up_col[wu] = (uint16_t)(j - s); up_val[wu] = v[q]; }
                        ++wu;
                    }
                }
            }
            carry_lo += __shfl_sync(0xffffffffu, il, 31);
            carry_up += __shfl_sync(0xffffffffu, iu, 31);
        }
        if (lane == 0) {
            lo_off[aps] = carry_lo;
            up_off[aps] = carry_up;
        }
        __syncwarp();
        if (lane == 0) {
            const bool ovl = carry_lo > p.cap_lo, ovu = carry_up > p.cap_up;
            if (want_lo) {
                for (int li = 0; li < aps; ++li) {
                    T acc = T(0);
                    if (!ovl) {
                        for (int q = lo_off[li]; q < lo_off[li + 1]; ++q)
                            acc = add_rn(acc, mul_rn(lo_val[q], ys[lo_col[q]]));
                    } else {
                        const int64_t i = s + li;
                        for (int q = rp[i]; q < rp[i + 1]; ++q) {
                            const int64_t j = ci[q];
                            if (j >= s && j < i) acc = add_rn(acc, mul_rn(v[q], ys[j - s]));
                        }
                    }
                    ys[li] = div_rn(sub_rn(ys[li], acc), ds[li]);
                }
            }
            if (SWEEP == 2)
                for (int li = 0; li < aps; ++li) ys[li] = mul_rn(ds[li], ys[li]);
            if (want_up) {
                for (int li = aps - 1; li >= 0; --li) {
                    T acc = T(0);
                    if (!ovu) {
                        for (int q = up_off[li]; q < up_off[li + 1]; ++q)
                            acc = add_rn(acc, mul_rn(up_val[q], ys[up_col[q]]));
                    } else {
                        const int64_t i = s + li;
                        for (int q = rp[i]; q < rp[i + 1]; ++q) {
                            const int64_t j = ci[q];
                            if (j > i && j <= e) acc = add_rn(acc, mul_rn(v[q], ys[j - s]));
                        }
                    }
                    ys[li] = div_rn(sub_rn(ys[li], acc), ds[li]);
                }
            }
        }
        __syncwarp();
        for (int li = lane; li < aps; li += 32) y[s + li] = (IO)ys[li];
        __syncwarp();
    }
}

template <typename T>
inline int dt_size() { return (int)sizeof(T); }
inline size_t dsize(int dt) { return dt == HS_F64 ? 8 : 4; }

}  // namespace

// ---------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------
struct hs_l1gs_s {
    int32_t n = 0, ps = 0, nparts = 0, ngroups = 0, nchunks = 0, chunksize = 0;
    int64_t npad = 0, tlen = 0, S = 0;
    int32_t sweep = 0, cache = 0, is_sym = 0, format = 0, mdt = 0, sdt = 0;
    double eta = 1.5;
    void* D = nullptr;
    void* Di = nullptr;
    void* SLi = nullptr;
    void* SUi = nullptr;
    int32_t* rp = nullptr;
    int32_t* ci = nullptr;
    void* vs = nullptr;
    int32_t cap_lo = 0, cap_up = 0;
    std::vector<int32_t> diag;
    alignas(64) CUtensorMap tmL;
    alignas(64) CUtensorMap tmU;
    void* dev_x = nullptr;
    void* dev_y = nullptr;
    int64_t bytes = 0;
    int E = 8, stages = 4;
};

namespace {

template <typename T>
int dmalloc(hs_l1gs* P, T** p, size_t bytes) {
    cudaError_t e = cudaMalloc((void**)p, bytes ? bytes : 1);
    if (e != cudaSuccess) return hs::cuda_error(e, "cudaMalloc");
    P->bytes += (int64_t)bytes;
    return HS_OK;
}

void release(hs_l1gs* P) {
    if (!P) return;
    void* ptrs[] = {P->D, P->Di, P->SLi, P->SUi, P->rp, P->ci, P->vs, P->dev_x, P->dev_y};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    delete P;
}

// Validate a host sparse matrix: sizes, monotone pointers, in-range and
// strictly ascending indices (a SparseMatrixCSC/CSR invariant).
int validate_sparse(const hs_sparse* A) {
    if (!A) return hs::set_error(HS_ERR_ARG, "matrix descriptor is NULL");
    if (A->n <= 0) return hs::set_error(HS_ERR_ARG, "matrix size must be greater than 0 (got %d)", A->n);
    if (A->format != HS_CSC && A->format != HS_CSR) return hs::set_error(HS_ERR_ARG, "unknown matrix format %d", A->format);
    if (A->dtype != HS_F64 && A->dtype != HS_F32) return hs::set_error(HS_ERR_ARG, "unknown value type %d", A->dtype);
    if (!A->ptr || (A->nnz > 0 && (!A->idx || !A->val))) return hs::set_error(HS_ERR_ARG, "matrix arrays are NULL");
    if (A->nnz < 0 || A->nnz > INT32_MAX) return hs::set_error(HS_ERR_ARG, "nnz out of range");
    if (A->ptr[0] != 0 || A->ptr[A->n] != A->nnz)
        return hs::set_error(HS_ERR_ARG, "pointer array must start at 0 and end at nnz");
    for (int32_t c = 0; c < A->n; ++c) {
        const int32_t a = A->ptr[c], b = A->ptr[c + 1];
        if (b < a) return hs::set_error(HS_ERR_ARG, "pointer array is not monotone at %d", c);
        for (int32_t q = a; q < b; ++q) {
            const int32_t r = A->idx[q];
            if (r < 0 || r >= A->n) return hs::set_error(HS_ERR_ARG, "index %d out of range at %d", r, q);
            if (q > a && A->idx[q - 1] >= r)
                return hs::set_error(HS_ERR_ARG, "indices must be strictly ascending within column/row %d", c);
        }
    }
    return HS_OK;
}

// DiagonalIndices (src/l1_gauss_seidel.jl:422-436) on the host.
template <typename TM>
int diag_indices(const hs_sparse* A, std::vector<int32_t>& diag) {
    const TM* val = static_cast<const TM*>(A->val);
    diag.resize(A->n);
    for (int32_t col = 0; col < A->n; ++col) {
        const int32_t r1 = A->ptr[col], r2 = A->ptr[col + 1] - 1;
        const int32_t* first = std::lower_bound(A->idx + r1, A->idx + r2 + 1, col);
        const int32_t pos = (int32_t)(first - A->idx);
        if (pos > r2 || A->idx[pos] != col || val[pos] == TM(0)) {
            hs::set_error(HS_ERR_SINGULAR, "SingularException(%d): missing or zero diagonal", col + 1);
            return hs::set_singular_col(col + 1);
        }
        diag[col] = pos;
    }
    return HS_OK;
}

// Stable CSC -> CSR transpose: iterating columns in order leaves every row's
// entries in ascending column order.
template <typename TM>
void transpose(const hs_sparse* A, std::vector<int32_t>& rp, std::vector<int32_t>& ci, std::vector<TM>& v) {
    const int32_t n = A->n;
    const TM* val = static_cast<const TM*>(A->val);
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
            v[cur[r]] = val[q];
            cur[r]++;
        }
}

template <typename TM, typename TS>
int setup_device(hs_l1gs* P, const int32_t* rp_h, const int32_t* ci_h, const TM* v_h, int64_t nnz,
                 cudaStream_t st) {
    const int32_t n = P->n;
    int32_t *rp_d = nullptr, *ci_d = nullptr;
    TM* v_d = nullptr;
    int rc;
    if ((rc = dmalloc(P, &rp_d, sizeof(int32_t) * (n + 1)))) return rc;
    P->rp = rp_d;
    if ((rc = dmalloc(P, &ci_d, sizeof(int32_t) * nnz))) return rc;
    P->ci = ci_d;
    if ((rc = dmalloc(P, &v_d, sizeof(TM) * nnz))) return rc;
    HS_CUDA(cudaMemcpyAsync(rp_d, rp_h, sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, st));
    HS_CUDA(cudaMemcpyAsync(ci_d, ci_h, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
    HS_CUDA(cudaMemcpyAsync(v_d, v_h, sizeof(TM) * nnz, cudaMemcpyHostToDevice, st));

    TS* D = nullptr;
    if ((rc = dmalloc(P, &D, sizeof(TS) * n))) return rc;
    P->D = D;
    TS *Di = nullptr, *SLi = nullptr, *SUi = nullptr;
    const bool packed = P->cache == HS_CACHE_PACKED;
    const bool lower = P->sweep != HS_SWEEP_BACKWARD, upper = P->sweep != HS_SWEEP_FORWARD;
    if (packed) {
        const int64_t dcount = (int64_t)P->ps * P->npad;
        if ((rc = dmalloc(P, &Di, sizeof(TS) * dcount))) return rc;
        P->Di = Di;
        fill_kernel<TS><<<std::min<int64_t>((dcount + 255) / 256, 4096), 256, 0, st>>>(Di, dcount, TS(1));
        HS_LAUNCH_CHECK("fill_kernel");
        const int64_t tcount = P->tlen * P->npad;
        if (lower && tcount > 0) {
            if ((rc = dmalloc(P, &SLi, sizeof(TS) * tcount))) return rc;
            P->SLi = SLi;
            HS_CUDA(cudaMemsetAsync(SLi, 0, sizeof(TS) * tcount, st));
        }
        if (upper && tcount > 0) {
            if ((rc = dmalloc(P, &SUi, sizeof(TS) * tcount))) return rc;
            P->SUi = SUi;
            HS_CUDA(cudaMemsetAsync(SUi, 0, sizeof(TS) * tcount, st));
        }
    }
    setup_rows_kernel<TM, TS><<<(n + 255) / 256, 256, 0, st>>>(n, P->ps, P->npad, rp_d, ci_d, v_d, (TM)P->eta, D,
                                                              Di, SLi, SUi);
    HS_LAUNCH_CHECK("setup_rows_kernel");
    if (packed) {
        HS_CUDA(cudaStreamSynchronize(st));
        cudaFree(rp_d);
        cudaFree(ci_d);
        cudaFree(v_d);
        P->bytes -= (int64_t)(sizeof(int32_t) * (n + 1 + nnz) + sizeof(TM) * nnz);
        P->rp = nullptr;
        P->ci = nullptr;
    } else {
        if (std::is_same<TM, TS>::value) {
            P->vs = v_d;
        } else {
            TS* vs = nullptr;
            if ((rc = dmalloc(P, &vs, sizeof(TS) * nnz))) return rc;
            convert_kernel<TM, TS><<<std::min<int64_t>((nnz + 255) / 256, 8192), 256, 0, st>>>(v_d, vs, nnz);
            HS_LAUNCH_CHECK("convert_kernel");
            HS_CUDA(cudaStreamSynchronize(st));
            cudaFree(v_d);
            P->bytes -= (int64_t)(sizeof(TM) * nnz);
            P->vs = vs;
        }
        // Shared-memory capacity: the largest in-block lower/upper count of any partition.
        int32_t ml = 0, mu = 0;
        for (int64_t k = 0; k < P->nparts; ++k) {
            const int64_t s = k * P->ps, e = std::min<int64_t>(s + P->ps - 1, n - 1);
            int32_t cl = 0, cu = 0;
            for (int64_t i = s; i <= e; ++i)
                for (int32_t q = rp_h[i]; q < rp_h[i + 1]; ++q) {
                    const int64_t j = ci_h[q];
                    cl += (j >= s && j < i);
                    cu += (j > i && j <= e);
                }
            ml = std::max(ml, cl);
            mu = std::max(mu, cu);
        }
        const int32_t limit = 4096;
        P->cap_lo = lower ? std::min(ml, limit) : 0;
        P->cap_up = upper ? std::min(mu, limit) : 0;
    }
    HS_CUDA(cudaStreamSynchronize(st));
    return HS_OK;
}

template <typename T, typename IO, int SWEEP, int E, int STAGES>
int launch_packed_t(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    PackedParams p;
    p.n = P->n;
    p.ps = P->ps;
    p.nparts = P->nparts;
    p.npad = P->npad;
    p.ngroups = P->ngroups;
    p.tlen = P->tlen;
    p.ntiles = (int32_t)((P->tlen + E - 1) / E);
    p.Di = P->Di;
    p.x = x;
    p.y = y;
    p.err = hs::device_error_word();
    p.ys_stride = 33;
    p.ring_bytes = (uint32_t)(E * 32 * sizeof(T) * STAGES);
    const uint32_t ys_bytes = (uint32_t)(P->ps * 33 * sizeof(T));
    p.warp_bytes = (p.ring_bytes + 8 * STAGES + ys_bytes + 127) / 128 * 128;
    const int wpb = (int)std::max<int64_t>(1, std::min<int64_t>(kWarpsPerBlock, (200 * 1024) / p.warp_bytes));
    const size_t smem = (size_t)p.warp_bytes * wpb;
    auto kern = l1gs_packed_kernel<T, IO, SWEEP, E, STAGES>;
    static thread_local int configured_smem = -1;
    if ((int)smem > configured_smem) {
        HS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured_smem = (int)smem;
    }
    int per_sm = 0;
    HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpb * 32, smem));
    if (per_sm < 1) return hs::set_error(HS_ERR_UNSUPPORTED, "partsize %d needs too much shared memory", P->ps);
    const int64_t want = (P->ngroups + wpb - 1) / wpb;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)per_sm * hs::num_sms()));
    kern<<<grid, wpb * 32, smem, st>>>(P->tmL, P->tmU, p);
    HS_LAUNCH_CHECK("l1gs_packed_kernel");
    return HS_OK;
}

template <typename T, typename IO, int SWEEP>
int launch_packed_cfg(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    constexpr int E = sizeof(T) == 8 ? 8 : 16;
    return launch_packed_t<T, IO, SWEEP, E, 4>(P, x, y, st);
}

template <typename T, typename IO, int SWEEP>
int launch_view_t(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    ViewParams p;
    p.n = P->n;
    p.ps = P->ps;
    p.nparts = P->nparts;
    p.rp = P->rp;
    p.ci = P->ci;
    p.v = P->vs;
    p.D = P->D;
    p.x = x;
    p.y = y;
    p.cap_lo = P->cap_lo;
    p.cap_up = P->cap_up;
    size_t b = sizeof(T) * (2 * (size_t)P->ps + p.cap_lo + p.cap_up) + sizeof(int32_t) * 2 * (P->ps + 1) +
               sizeof(uint16_t) * (p.cap_lo + p.cap_up);
    p.warp_bytes = (uint32_t)((b + 15) / 16 * 16);
    const int wpb = (int)std::max<int64_t>(1, std::min<int64_t>(kWarpsPerBlock, (200 * 1024) / p.warp_bytes));
    const size_t smem = (size_t)p.warp_bytes * wpb;
    auto kern = l1gs_view_kernel<T, IO, SWEEP>;
    static thread_local int configured_smem = -1;
    if ((int)smem > configured_smem) {
        HS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured_smem = (int)smem;
    }
    int per_sm = 0;
    HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpb * 32, smem));
    if (per_sm < 1) return hs::set_error(HS_ERR_UNSUPPORTED, "view partition needs too much shared memory");
    const int64_t want = (P->nparts + wpb - 1) / wpb;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)per_sm * hs::num_sms()));
    kern<<<grid, wpb * 32, smem, st>>>(p);
    HS_LAUNCH_CHECK("l1gs_view_kernel");
    return HS_OK;
}

template <typename T, typename IO>
int launch_apply(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    if (P->cache == HS_CACHE_PACKED) {
        switch (P->sweep) {
            case HS_SWEEP_FORWARD: return launch_packed_cfg<T, IO, 0>(P, x, y, st);
            case HS_SWEEP_BACKWARD: return launch_packed_cfg<T, IO, 1>(P, x, y, st);
            default: return launch_packed_cfg<T, IO, 2>(P, x, y, st);
        }
    }
    switch (P->sweep) {
        case HS_SWEEP_FORWARD: return launch_view_t<T, IO, 0>(P, x, y, st);
        case HS_SWEEP_BACKWARD: return launch_view_t<T, IO, 1>(P, x, y, st);
        default: return launch_view_t<T, IO, 2>(P, x, y, st);
    }
}

template <typename TS>
void unpack_reference(const hs_l1gs* P, const TS* inter, TS* out, bool lower) {
    const int64_t ps = P->ps, tlen = P->tlen;
    for (int64_t k = 0; k < P->nparts; ++k) {
        const int64_t s = k * ps, e = std::min<int64_t>(s + ps - 1, P->n - 1), aps = e - s + 1;
        const int64_t boff = k * tlen;
        for (int64_t li = 0; li < aps; ++li) {
            if (lower) {
                for (int64_t lj = 0; lj < li; ++lj)
                    out[boff + li * (li - 1) / 2 + lj] = inter[lo_idx(li, lj) * P->npad + k];
            } else {
                const int64_t row_start = li * aps - li * (li + 1) / 2;
                for (int64_t lj = li + 1; lj < aps; ++lj)
                    out[boff + row_start + (lj - li) - 1] = inter[up_idx(ps, li, lj) * P->npad + k];
            }
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int hs_l1gs_create(const hs_sparse* A, int32_t partsize, int32_t is_sym, double eta, int32_t sweep, int32_t cache,
                   int32_t smoother_dtype, int32_t threads, int32_t blocks, void* stream, hs_l1gs** out) {
    if (!out) return hs::set_error(HS_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (partsize <= 0) return hs::set_error(HS_ERR_ARG, "partsize must be greater than 0");
    if (threads <= 0) return hs::set_error(HS_ERR_ARG, "`threads` must be greater than 0");
    if (blocks <= 0) return hs::set_error(HS_ERR_ARG, "`blocks` must be greater than 0");
    if (sweep < 0 || sweep > 2) return hs::set_error(HS_ERR_ARG, "unknown sweep %d", sweep);
    if (cache != HS_CACHE_PACKED && cache != HS_CACHE_VIEW) return hs::set_error(HS_ERR_ARG, "unknown cache %d", cache);
    if (smoother_dtype != HS_F64 && smoother_dtype != HS_F32)
        return hs::set_error(HS_ERR_ARG, "unknown smoother dtype %d", smoother_dtype);
    int rc = validate_sparse(A);
    if (rc) return rc;
    if (A->dtype == HS_F32 && smoother_dtype == HS_F64)
        return hs::set_error(HS_ERR_UNSUPPORTED, "an FP64 smoother needs an FP64 matrix");
    if (partsize > 65535) return hs::set_error(HS_ERR_UNSUPPORTED, "partsize above 65535");

    hs_l1gs* P = new hs_l1gs();
    P->n = A->n;
    P->ps = partsize;
    P->nparts = (int32_t)(((int64_t)A->n + partsize - 1) / partsize);
    P->npad = ((int64_t)P->nparts + 31) / 32 * 32;
    P->ngroups = (int32_t)(P->npad / 32);
    P->tlen = (int64_t)partsize * (partsize - 1) / 2;
    const int64_t lps = (int64_t)A->n - (int64_t)(P->nparts - 1) * partsize;
    P->S = P->tlen * (P->nparts - 1) + lps * (lps - 1) / 2;
    P->nchunks = blocks;  // _blockpartitioning for KA.GPU (:353-365)
    P->chunksize = (int32_t)std::min<int64_t>(((int64_t)P->nparts + blocks - 1) / blocks, threads);
    P->sweep = sweep;
    P->cache = cache;
    P->is_sym = is_sym ? 1 : 0;
    P->format = A->format;
    P->mdt = A->dtype;
    P->sdt = smoother_dtype;
    P->eta = eta;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Row i of the preconditioner is read from: the CSR row; column i of a
    // CSC when isSymA (:1218-1229); the true row of a non-symmetric CSC,
    // after DiagonalIndices validated the diagonal (:619, :422-436).
    std::vector<int32_t> trp, tci;
    std::vector<double> tv64;
    std::vector<float> tv32;
    const int32_t* rp_h = A->ptr;
    const int32_t* ci_h = A->idx;
    const void* v_h = A->val;
    if (A->format == HS_CSC && !is_sym) {
        rc = A->dtype == HS_F64 ? diag_indices<double>(A, P->diag) : diag_indices<float>(A, P->diag);
        if (rc) {
            release(P);
            return rc;
        }
        if (A->dtype == HS_F64) {
            transpose<double>(A, trp, tci, tv64);
            v_h = tv64.data();
        } else {
            transpose<float>(A, trp, tci, tv32);
            v_h = tv32.data();
        }
        rp_h = trp.data();
        ci_h = tci.data();
    }

    if (A->dtype == HS_F64 && smoother_dtype == HS_F64)
        rc = setup_device<double, double>(P, rp_h, ci_h, static_cast<const double*>(v_h), A->nnz, st);
    else if (A->dtype == HS_F64)
        rc = setup_device<double, float>(P, rp_h, ci_h, static_cast<const double*>(v_h), A->nnz, st);
    else
        rc = setup_device<float, float>(P, rp_h, ci_h, static_cast<const float*>(v_h), A->nnz, st);
    if (rc) {
        release(P);
        return rc;
    }
    if (cache == HS_CACHE_PACKED) {
        const uint32_t E = smoother_dtype == HS_F64 ? 8 : 16;
        const void* l = P->SLi ? P->SLi : P->SUi;
        const void* u = P->SUi ? P->SUi : P->SLi;
        if (l) {
            const size_t es = dsize(smoother_dtype);
            if ((rc = hs::encode_tensor_map_2d(&P->tmL, l, smoother_dtype, P->npad, P->tlen, P->npad * es, 32, E)) ||
                (rc = hs::encode_tensor_map_2d(&P->tmU, u, smoother_dtype, P->npad, P->tlen, P->npad * es, 32, E))) {
                release(P);
                return rc;
            }
        } else {
            std::memset(&P->tmL, 0, sizeof(CUtensorMap));
            std::memset(&P->tmU, 0, sizeof(CUtensorMap));
        }
    }
    *out = P;
    return HS_OK;
}

int hs_l1gs_apply(hs_l1gs* P, const void* x, void* y, int32_t io_dtype, void* stream) {
    if (!P || !x || !y) return hs::set_error(HS_ERR_ARG, "hs_l1gs_apply: NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (P->sdt == HS_F64 && io_dtype == HS_F64) return launch_apply<double, double>(P, x, y, st);
    if (P->sdt == HS_F32 && io_dtype == HS_F32) return launch_apply<float, float>(P, x, y, st);
    if (P->sdt == HS_F32 && io_dtype == HS_F64) return launch_apply<float, double>(P, x, y, st);
    return hs::set_error(HS_ERR_UNSUPPORTED, "FP64 smoother with FP32 vectors is not provided");
}

int hs_l1gs_apply_host(hs_l1gs* P, const void* x_host, void* y_host, int32_t io_dtype, void* stream) {
    if (!P || !x_host || !y_host) return hs::set_error(HS_ERR_ARG, "hs_l1gs_apply_host: NULL argument");
    const size_t bytes = dsize(io_dtype) * (size_t)P->n;
    if (!P->dev_x) {
        int rc;
        if ((rc = dmalloc(P, &P->dev_x, bytes))) return rc;
        if ((rc = dmalloc(P, &P->dev_y, bytes))) return rc;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    HS_CUDA(cudaMemcpyAsync(P->dev_x, x_host, bytes, cudaMemcpyHostToDevice, st));
    int rc = hs_l1gs_apply(P, P->dev_x, P->dev_y, io_dtype, stream);
    if (rc) return rc;
    HS_CUDA(cudaMemcpyAsync(y_host, P->dev_y, bytes, cudaMemcpyDeviceToHost, st));
    HS_CUDA(cudaStreamSynchronize(st));
    return HS_OK;
}

int hs_l1gs_info_get(const hs_l1gs* P, hs_l1gs_info* info) {
    if (!P || !info) return hs::set_error(HS_ERR_ARG, "hs_l1gs_info_get: NULL argument");
    info->n = P->n;
    info->partsize = P->ps;
    info->nparts = P->nparts;
    info->nchunks = P->nchunks;
    info->chunksize = P->chunksize;
    info->sweep = P->sweep;
    info->cache = P->cache;
    info->is_sym = P->is_sym;
    info->format = P->format;
    info->matrix_dtype = P->mdt;
    info->smoother_dtype = P->sdt;
    info->packed_len = P->S;
    info->device_bytes = P->bytes;
    info->eta = P->eta;
    return HS_OK;
}

int hs_l1gs_get_diag(const hs_l1gs* P, void* out_host) {
    if (!P || !out_host) return hs::set_error(HS_ERR_ARG, "hs_l1gs_get_diag: NULL argument");
    HS_CUDA(cudaDeviceSynchronize());
    HS_CUDA(cudaMemcpy(out_host, P->D, dsize(P->sdt) * P->n, cudaMemcpyDeviceToHost));
    return HS_OK;
}

int hs_l1gs_get_packed(const hs_l1gs* P, int32_t which, void* out_host, int64_t capacity) {
    if (!P || !out_host) return hs::set_error(HS_ERR_ARG, "hs_l1gs_get_packed: NULL argument");
    if (P->cache != HS_CACHE_PACKED) return hs::set_error(HS_ERR_ARG, "not a packed-cache preconditioner");
    const void* src = which == 0 ? P->SLi : P->SUi;
    const bool has = which == 0 ? P->sweep != HS_SWEEP_BACKWARD : P->sweep != HS_SWEEP_FORWARD;
    if (!has) return hs::set_error(HS_ERR_ARG, "this sweep has no %s buffer", which == 0 ? "SL" : "SU");
    if (capacity < P->S) return hs::set_error(HS_ERR_ARG, "capacity %lld < %lld", (long long)capacity, (long long)P->S);
    const size_t es = dsize(P->sdt);
    std::memset(out_host, 0, es * P->S);
    if (!src) return HS_OK;  // partsize 1: empty triangles
    std::vector<unsigned char> inter(es * P->tlen * P->npad);
    HS_CUDA(cudaDeviceSynchronize());
    HS_CUDA(cudaMemcpy(inter.data(), src, inter.size(), cudaMemcpyDeviceToHost));
    if (P->sdt == HS_F64)
        unpack_reference<double>(P, reinterpret_cast<const double*>(inter.data()), static_cast<double*>(out_host),
                                 which == 0);
    else
        unpack_reference<float>(P, reinterpret_cast<const float*>(inter.data()), static_cast<float*>(out_host),
                                which == 0);
    return HS_OK;
}

int hs_l1gs_get_diag_indices(const hs_l1gs* P, int32_t* out_host) {
    if (!P || !out_host) return hs::set_error(HS_ERR_ARG, "hs_l1gs_get_diag_indices: NULL argument");
    if (P->diag.empty()) return hs::set_error(HS_ERR_ARG, "DiagonalIndices exist only for non-symmetric CSC input");
    std::memcpy(out_host, P->diag.data(), sizeof(int32_t) * P->diag.size());
    return HS_OK;
}

int hs_l1gs_destroy(hs_l1gs* P) {
    if (P) cudaDeviceSynchronize();
    release(P);
    return HS_OK;
}

}  // extern "C"
