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
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "l1gs_coop.cuh"
#include "l1gs_seg.cuh"

namespace {

constexpr int kWarpsPerBlock = 4;

__host__ __device__ __forceinline__ int64_t lo_idx(int64_t li, int64_t lj) { return li * (li - 1) / 2 + lj; }
__host__ __device__ __forceinline__ int64_t up_idx(int64_t ps, int64_t li, int64_t lj) {
    int64_t q = ps - 1 - li;
    return q * (q - 1) / 2 + (lj - li - 1);
}

// Row-aligned stream layout for partsize >= 32 ("rows" layout) with tile
// width e (8 or 32 slots).  Row r of a direction (r = li forward, r = ps-1-li
// backward) occupies r + 1 slots rounded up to a multiple of e, from
// rows_off(r, e): slot 0 holds D_Dl1 of the row, slots 1.. its terms in the
// order the sweep sums them, then zeros.  Every tile belongs to one row, so
// the apply streams whole tiles with a fixed-length inner loop and receives
// D_Dl1 with the row's first tile.
__host__ __device__ __forceinline__ int64_t rows_off(int64_t r, int64_t e) {   // sum_{u=1..r} of u rounded up to e
    const int64_t m = r / e, rem = r % e;
    return e * e * m * (m + 1) / 2 + e * (m + 1) * rem;
}

// ---------------------------------------------------------------------------
// Setup: D_Dl1 and packing, one thread per row.
//   D_Dl1: _diag_offpart_rowwise (:1101-1129) + eta rule (:1017-1022)
//   packing: _pack_strict_lower/upper_rowwise! (:1248-1277, :1380-1413)
// TM is the matrix value type (the type D_Dl1 is computed in), TS the
// smoother type it is stored in.
// ---------------------------------------------------------------------------
// With a cooperative layout (coop.G > 0) the triangles go to SC instead, in
// the column-block order of l1gs_coop.cuh (coop_dirs: 1 lower, 2 upper).
template <typename TM, typename TS>
__global__ void setup_rows_kernel(int32_t n, int32_t ps, int64_t npad, const int32_t* __restrict__ rp,
                                  const int32_t* __restrict__ ci, const TM* __restrict__ v, TM eta,
                                  TS* __restrict__ D, TS* __restrict__ Di, TS* __restrict__ SLi,
                                  TS* __restrict__ SUi, int rows_layout, hscoop::Layout coop, int coop_dirs,
                                  TS* __restrict__ SC) {
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
            if (SC) {
                if (coop_dirs & 1) SC[hscoop::lower_idx(coop, k, li, j - s)] = (TS)val;
            } else if (SLi) {
                SLi[(rows_layout ? rows_off(li, rows_layout) + 1 + (j - s) : lo_idx(li, j - s)) * npad + k] = (TS)val;
            }
        } else {
            if (SC) {
                if (coop_dirs & 2) SC[hscoop::upper_idx(coop, k, li, j - s)] = (TS)val;
            } else if (SUi) {
                SUi[(rows_layout ? rows_off(ps - 1 - li, rows_layout) + (j - i) : up_idx(ps, li, j - s)) * npad + k] =
                    (TS)val;
            }
        }
    }
    const TM dl1star = (b >= mul_rn(eta, d)) ? TM(0) : div_rn(d, TM(2));
    const TM Dv = add_rn(b, dl1star);
    D[i] = (TS)Dv;
    if (Di) Di[li * npad + k] = (TS)Dv;
    if (rows_layout) {
        if (SLi) SLi[rows_off(li, rows_layout) * npad + k] = (TS)Dv;
        if (SUi) SUi[rows_off(ps - 1 - li, rows_layout) * npad + k] = (TS)Dv;
    }
}

// Rows layout: the missing rows of a short last partition get D_Dl1 = 1 in
// their stream slots (their y stays 0 and adds +0.0 terms only).
template <typename TS>
__global__ void rows_tail_kernel(int32_t ps, int32_t lps, int64_t npad, int64_t k, int32_t e, TS* __restrict__ SLi,
                                 TS* __restrict__ SUi) {
    for (int li = lps + threadIdx.x; li < ps; li += blockDim.x) {
        if (SLi) SLi[rows_off(li, e) * npad + k] = TS(1);
        if (SUi) SUi[rows_off(ps - 1 - li, e) * npad + k] = TS(1);
    }
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
//
// Each warp walks its groups g = g0, g0+gstride, ... (32 partitions each) and
// consumes, per group, the lower stream then/or the upper stream as tiles of
// E rows x 32 lanes.  Tile t of the warp's whole sequence lives in ring stage
// t % STAGES; lane 0 refills a stage with tile t+STAGES as soon as the warp has
// read tile t, so STAGES-1 tiles are always in flight, across group
// boundaries too.  Every wait is bounded; on a timeout the warp records
// kErrWaitTimeout, lets its in-flight copies land (bounded) and returns.
// ---------------------------------------------------------------------------
struct PackedParams {
    int32_t n, ps, nparts;
    int64_t npad;
    int32_t gbeg, ngroups;   // groups [gbeg, ngroups) of this launch
    int32_t tlen;      // ps(ps-1)/2 stream elements per direction
    int32_t ntiles;    // ceil(tlen / E) tiles per direction
    const void* Di;
    const void* x;
    void* y;
    int32_t* err;
    uint32_t warp_bytes;
    uint32_t ring_bytes;
};

template <typename T, int E, int STAGES, int SWEEP>
struct TileRing {
    const CUtensorMap* tmL;
    const CUtensorMap* tmU;
    T* buf;
    uint64_t* bars;
    int32_t g0, gstride, ntiles, total;
    int lane;
    mutable int32_t last = 0;   // the tile of the latest wait (a timeout drains from here)

    __device__ __forceinline__ void issue(int32_t c) const {
        const int32_t ntpg = (SWEEP == 2) ? 2 * ntiles : ntiles;
        const int32_t gi = c / ntpg;
        int32_t ti = c - gi * ntpg;
        const CUtensorMap* map = (SWEEP == 1) ? tmU : tmL;
        if (SWEEP == 2 && ti >= ntiles) {
            map = tmU;
            ti -= ntiles;
        }
        const int stage = c & (STAGES - 1);
        hsdev::mbar_arrive_expect_tx(bars + stage, (uint32_t)(E * 32 * sizeof(T)));
        hsdev::tma_load_2d(buf + stage * (E * 32), map, (g0 + gi * gstride) * 32, ti * E, bars + stage);
    }
    __device__ __forceinline__ void prologue() const {
        if (lane == 0) {
            for (int s = 0; s < STAGES; ++s) hsdev::mbar_init(bars + s, 1);
            hsdev::fence_barrier_init();
            const int32_t pro = total < STAGES ? total : STAGES;
            for (int32_t c = 0; c < pro; ++c) issue(c);
        }
        __syncwarp();
    }
    // Wait for tile c; false (on every lane) if a bounded wait ran out.
    __device__ __forceinline__ bool wait(int32_t c) const {
        last = c;
        const bool ok = hsdev::mbar_wait_bounded(bars + (c & (STAGES - 1)), (uint32_t)((c / STAGES) & 1));
        return __all_sync(0xffffffffu, ok);
    }
    __device__ __forceinline__ const T* tile(int32_t c) const { return buf + (c & (STAGES - 1)) * (E * 32); }
    // The warp has read tile c: refill its stage with tile c+STAGES.
    __device__ __forceinline__ void release(int32_t c) const {
        __syncwarp();
        if (lane == 0 && c + STAGES < total) {
            hsdev::fence_proxy_async_smem();
            issue(c + STAGES);
        }
    }
    // After a timeout: let the copies issued for the tiles from the one that
    // timed out on (at most STAGES of them) land, then return.
    __device__ void drain(int32_t /*unused*/, int32_t* err) const {
        if (lane == 0) hsdev::report_error(err, hsdev::kErrWaitTimeout);
        const int32_t c = last;
        const int32_t end = (c + STAGES < total) ? c + STAGES : total;
        for (int32_t cc = c; cc < end; ++cc)
            (void)hsdev::mbar_wait_bounded(bars + (cc & (STAGES - 1)), (uint32_t)((cc / STAGES) & 1));
    }
};

// ---- compile-time partsize: y and D_Dl1 in registers, fully unrolled -------
template <typename T, typename IO, int SWEEP, int PS, int E, int STAGES, int MINB>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, MINB)
    l1gs_packed_small_kernel(const __grid_constant__ CUtensorMap tmL, const __grid_constant__ CUtensorMap tmU,
                             const PackedParams p) {
    constexpr int TLEN = PS * (PS - 1) / 2;
    constexpr int NT = (TLEN + E - 1) / E;
    constexpr int XS = (PS % 2 == 0) ? PS + 1 : PS;  // odd stride: conflict-free transposes
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    unsigned char* wbase = smem + (size_t)warp * p.warp_bytes;
    T* xs = reinterpret_cast<T*>(wbase + p.ring_bytes + 8 * STAGES);
    const T* __restrict__ Di = static_cast<const T*>(p.Di);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);

    const int wpb = blockDim.x >> 5;
    TileRing<T, E, STAGES, SWEEP> ring;
    ring.tmL = &tmL;
    ring.tmU = &tmU;
    ring.buf = reinterpret_cast<T*>(wbase);
    ring.bars = reinterpret_cast<uint64_t*>(wbase + p.ring_bytes);
    ring.g0 = p.gbeg + blockIdx.x * wpb + warp;
    ring.gstride = gridDim.x * wpb;
    ring.ntiles = NT;
    ring.lane = lane;
    const int32_t my_groups = ring.g0 < p.ngroups ? (p.ngroups - 1 - ring.g0) / ring.gstride + 1 : 0;
    ring.total = my_groups * ((SWEEP == 2) ? 2 * NT : NT);
    if (NT > 0) ring.prologue();

    int32_t c = 0;  // first tile of the current direction
    for (int32_t gi = 0; gi < my_groups; ++gi) {
        const int64_t g = ring.g0 + (int64_t)gi * ring.gstride;
        const int64_t k = g * 32 + lane;
        const int64_t rowbase = g * 32 * PS;
        T d[PS];
#pragma unroll
        for (int li = 0; li < PS; ++li) d[li] = Di[(int64_t)li * p.npad + k];
#pragma unroll
        for (int m = 0; m < PS; ++m) {
            const int t = lane + 32 * m;
            const int64_t row = rowbase + t;
            xs[(t / PS) * XS + (t % PS)] = row < p.n ? (T)x[row] : T(0);
        }
        __syncwarp();
        T yv[PS];
#pragma unroll
        for (int li = 0; li < PS; ++li) yv[li] = xs[lane * XS + li];

        if (SWEEP != 1) {  // forward: rows ascending, lower stream e = li(li-1)/2 + lj
#pragma unroll
            for (int li = 0; li < PS; ++li) {
                T acc = T(0);
#pragma unroll
                for (int lj = 0; lj < li; ++lj) {
                    const int e = li * (li - 1) / 2 + lj;
                    if (e % E == 0 && !ring.wait(c + e / E)) goto timeout;
                    acc = add_rn(acc, mul_rn(ring.tile(c + e / E)[(e % E) * 32 + lane], yv[lj]));
                    if (e % E == E - 1 || e == TLEN - 1) ring.release(c + e / E);
                }
                yv[li] = div_rn(sub_rn(yv[li], acc), d[li]);
            }
            c += NT;
        }
        if (SWEEP == 2) {  // y .= D_Dl1 .* y  (:897)
#pragma unroll
            for (int li = 0; li < PS; ++li) yv[li] = mul_rn(d[li], yv[li]);
        }
        if (SWEEP != 0) {  // backward: rows descending, upper stream e = q(q-1)/2 + (lj-li-1)
#pragma unroll
            for (int li = PS - 1; li >= 0; --li) {
                T acc = T(0);
#pragma unroll
                for (int lj = li + 1; lj < PS; ++lj) {
                    const int q = PS - 1 - li;
                    const int e = q * (q - 1) / 2 + (lj - li - 1);
                    if (e % E == 0 && !ring.wait(c + e / E)) goto timeout;
                    acc = add_rn(acc, mul_rn(ring.tile(c + e / E)[(e % E) * 32 + lane], yv[lj]));
                    if (e % E == E - 1 || e == TLEN - 1) ring.release(c + e / E);
                }
                yv[li] = div_rn(sub_rn(yv[li], acc), d[li]);
            }
            c += NT;
        }
        __syncwarp();
#pragma unroll
        for (int li = 0; li < PS; ++li) xs[lane * XS + li] = yv[li];
        __syncwarp();
#pragma unroll
        for (int m = 0; m < PS; ++m) {
            const int t = lane + 32 * m;
            const int64_t row = rowbase + t;
            if (row < p.n) y[row] = (IO)xs[(t / PS) * XS + (t % PS)];
        }
        __syncwarp();
    }
    return;
timeout:
    ring.drain(c, p.err);
}

// ---- runtime partsize: y in shared memory, tile-major stream walk ---------
template <typename T, typename IO, int SWEEP, int E, int STAGES>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    l1gs_packed_kernel(const __grid_constant__ CUtensorMap tmL, const __grid_constant__ CUtensorMap tmU,
                       const PackedParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int S = 33;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    unsigned char* wbase = smem + (size_t)warp * p.warp_bytes;
    T* ys = reinterpret_cast<T*>(wbase + p.ring_bytes + 8 * STAGES);
    const T* __restrict__ Di = static_cast<const T*>(p.Di);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);
    const int ps = p.ps;

    const int wpb = blockDim.x >> 5;
    TileRing<T, E, STAGES, SWEEP> ring;
    ring.tmL = &tmL;
    ring.tmU = &tmU;
    ring.buf = reinterpret_cast<T*>(wbase);
    ring.bars = reinterpret_cast<uint64_t*>(wbase + p.ring_bytes);
    ring.g0 = p.gbeg + blockIdx.x * wpb + warp;
    ring.gstride = gridDim.x * wpb;
    ring.ntiles = p.ntiles;
    ring.lane = lane;
    const int32_t my_groups = ring.g0 < p.ngroups ? (p.ngroups - 1 - ring.g0) / ring.gstride + 1 : 0;
    ring.total = my_groups * ((SWEEP == 2) ? 2 * p.ntiles : p.ntiles);
    if (p.ntiles > 0) ring.prologue();

    int32_t c = 0;
    for (int32_t gi = 0; gi < my_groups; ++gi) {
        const int64_t g = ring.g0 + (int64_t)gi * ring.gstride;
        const int64_t k = g * 32 + lane;
        const int64_t rowbase = g * 32 * (int64_t)ps;
        const T* __restrict__ dk = Di + k;   // D_Dl1 of row li at dk[li * npad]
        T* yk = ys + lane;                   // y of row li at yk[li * S]
        for (int t = lane; t < 32 * ps; t += 32) {
            const int64_t row = rowbase + t;
            ys[(t % ps) * S + t / ps] = row < p.n ? (T)x[row] : T(0);
        }
        __syncwarp();

        if (SWEEP != 1) {  // forward: rows ascending over the lower stream
            T dnext = dk[(ps > 1 ? 1 : 0) * p.npad];
            yk[0] = div_rn(sub_rn(yk[0], T(0)), dk[0]);
            int32_t t = 0, r = 0;
            for (int li = 1; li < ps; ++li) {
                const T dcur = dnext;
                if (li + 1 < ps) dnext = dk[(int64_t)(li + 1) * p.npad];
                T acc = T(0);
                int lj = 0;
                while (lj < li) {
                    if (r == 0 && !ring.wait(c + t)) goto timeout;
                    const T* tl = ring.tile(c + t) + r * 32 + lane;
                    const int cnt = min(li - lj, E - r);
                    for (int b0 = 0; b0 < cnt; b0 += 8) {
                        T av[8], yv[8];
#pragma unroll
                        for (int m = 0; m < 8; ++m)
                            if (b0 + m < cnt) {
                                av[m] = tl[(b0 + m) * 32];
                                yv[m] = yk[(lj + b0 + m) * S];
                            }
#pragma unroll
                        for (int m = 0; m < 8; ++m)
                            if (b0 + m < cnt) acc = add_rn(acc, mul_rn(av[m], yv[m]));
                    }
                    lj += cnt;
                    r += cnt;
                    if (r == E) {
                        ring.release(c + t);
                        ++t;
                        r = 0;
                    }
                }
                yk[li * S] = div_rn(sub_rn(yk[li * S], acc), dcur);
            }
            if (r != 0) ring.release(c + t);
            c += p.ntiles;
        }
        if (SWEEP == 2) {
            for (int li = 0; li < ps; ++li) yk[li * S] = mul_rn(dk[(int64_t)li * p.npad], yk[li * S]);
        }
        if (SWEEP != 0) {  // backward: rows descending over the upper stream
            T dnext = dk[(int64_t)(ps > 1 ? ps - 2 : 0) * p.npad];
            yk[(ps - 1) * S] = div_rn(sub_rn(yk[(ps - 1) * S], T(0)), dk[(int64_t)(ps - 1) * p.npad]);
            int32_t t = 0, r = 0;
            for (int li = ps - 2; li >= 0; --li) {
                const T dcur = dnext;
                if (li > 0) dnext = dk[(int64_t)(li - 1) * p.npad];
                T acc = T(0);
                int lj = li + 1;
                while (lj < ps) {
                    if (r == 0 && !ring.wait(c + t)) goto timeout;
                    const T* tl = ring.tile(c + t) + r * 32 + lane;
                    const int cnt = min(ps - lj, E - r);
                    for (int b0 = 0; b0 < cnt; b0 += 8) {
                        T av[8], yv[8];
#pragma unroll
                        for (int m = 0; m < 8; ++m)
                            if (b0 + m < cnt) {
                                av[m] = tl[(b0 + m) * 32];
                                yv[m] = yk[(lj + b0 + m) * S];
                            }
#pragma unroll
                        for (int m = 0; m < 8; ++m)
                            if (b0 + m < cnt) acc = add_rn(acc, mul_rn(av[m], yv[m]));
                    }
                    lj += cnt;
                    r += cnt;
                    if (r == E) {
                        ring.release(c + t);
                        ++t;
                        r = 0;
                    }
                }
                yk[li * S] = div_rn(sub_rn(yk[li * S], acc), dcur);
            }
            if (r != 0) ring.release(c + t);
            c += p.ntiles;
        }
        __syncwarp();
        for (int t = lane; t < 32 * ps; t += 32) {
            const int64_t row = rowbase + t;
            if (row < p.n) y[row] = (IO)ys[(t % ps) * S + t / ps];
        }
        __syncwarp();
    }
    return;
timeout:
    ring.drain(c, p.err);
}

// Shared-memory loads issued in program order: a tile's coefficient and y
// loads all go out before its multiply-adds, so one warp per SM sub-partition
// (large partsizes have few partitions) waits for them once per 8 slots.
__device__ __forceinline__ double lds_t(const double* p) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(hsdev::smem_u32(p)) : "memory");
    return v;
}
__device__ __forceinline__ float lds_t(const float* p) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(hsdev::smem_u32(p)) : "memory");
    return v;
}

// A row's running sum.  NACC = 1: one sum in the order the terms arrive --
// ascending column, the reference's order, bit-identical.  NACC = 4: the term
// in tile slot m goes to partial sum m % 4 and the row's total is
// (s0 + s1) + (s2 + s3); four independent add chains instead of one, a
// different rounding (relative 1e-12 of the reference in FP64).
template <typename T, int NACC>
struct RowAcc;
template <typename T>
struct RowAcc<T, 1> {
    T a = T(0);
    __device__ __forceinline__ void add(int, T p) { a = add_rn(a, p); }
    __device__ __forceinline__ T total() const { return a; }
};
template <typename T>
struct RowAcc<T, 4> {
    T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
    __device__ __forceinline__ void add(int m, T p) {   // m is a compile-time slot index after unrolling
        switch (m & 3) {
            case 0: a0 = add_rn(a0, p); break;
            case 1: a1 = add_rn(a1, p); break;
            case 2: a2 = add_rn(a2, p); break;
            default: a3 = add_rn(a3, p); break;
        }
    }
    __device__ __forceinline__ T total() const { return add_rn(add_rn(a0, a1), add_rn(a2, a3)); }
};

// acc += sum_{m<8} tl[m*32] * yy[m*S] in slot order, loads first.
template <typename T, int S, typename ACC>
__device__ __forceinline__ void fold8(ACC& acc, const T* tl, const T* yy) {
    T a[8], b[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        a[m] = lds_t(tl + m * 32);
        b[m] = lds_t(yy + m * S);
    }
#pragma unroll
    for (int m = 0; m < 8; ++m) acc.add(m, mul_rn(a[m], b[m]));
}

// Ring for the rows kernel: like TileRing, but the elected lane keeps the
// coordinates of the next tile to fetch and advances them by one per refill
// (no division per tile: a refill is a few instructions).
template <typename T, int E, int STAGES, int SWEEP>
struct RowRing {
    const CUtensorMap* tmL;
    const CUtensorMap* tmU;
    T* buf;
    uint64_t* bars;
    int32_t total, ntiles, gstride;
    int lane;
    int32_t issued = 0, i_g = 0, i_ti = 0, i_dir = 0;   // next tile to fetch (elected lane)
    mutable int32_t last = 0;

    __device__ __forceinline__ void issue_next() {
        const int stage = issued & (STAGES - 1);
        const CUtensorMap* map = (SWEEP == 1 || (SWEEP == 2 && i_dir)) ? tmU : tmL;
        hsdev::mbar_arrive_expect_tx(bars + stage, (uint32_t)(E * 32 * sizeof(T)));
        hsdev::tma_load_2d(buf + stage * (E * 32), map, i_g * 32, i_ti * E, bars + stage);
        ++issued;
        if (++i_ti == ntiles) {
            i_ti = 0;
            if (SWEEP == 2 && !i_dir) {
                i_dir = 1;
            } else {
                i_dir = 0;
                i_g += gstride;
            }
        }
    }
    __device__ __forceinline__ void prologue(int32_t g0) {
        if (lane == 0) {
            i_g = g0;
            for (int s = 0; s < STAGES; ++s) hsdev::mbar_init(bars + s, 1);
            hsdev::fence_barrier_init();
            const int32_t pro = total < STAGES ? total : STAGES;
            for (int32_t c = 0; c < pro; ++c) issue_next();
        }
        __syncwarp();
    }
    __device__ __forceinline__ bool wait(int32_t c) const {
        last = c;
        const bool ok = hsdev::mbar_wait_bounded(bars + (c & (STAGES - 1)), (uint32_t)((c / STAGES) & 1));
        return __all_sync(0xffffffffu, ok);
    }
    __device__ __forceinline__ const T* tile(int32_t c) const { return buf + (c & (STAGES - 1)) * (E * 32); }
    __device__ __forceinline__ void release(int32_t c) {
        __syncwarp();
        if (lane == 0 && c + STAGES < total) {
            hsdev::fence_proxy_async_smem();
            issue_next();
        }
    }
    __device__ void drain(int32_t* err) const {
        if (lane == 0) hsdev::report_error(err, hsdev::kErrWaitTimeout);
        const int32_t c = last;
        const int32_t end = (c + STAGES < total) ? c + STAGES : total;
        for (int32_t cc = c; cc < end; ++cc)
            (void)hsdev::mbar_wait_bounded(bars + (cc & (STAGES - 1)), (uint32_t)((cc / STAGES) & 1));
    }
};

// ---- partsize >= 32: row-aligned streams (rows layout) ----------------------
// Thread per partition as above.  Each row's stream segment starts with its
// D_Dl1 and is padded to whole 8-slot tiles, so a full tile is 8 loads of
// coefficients, 8 of y and 8 separately rounded multiply-adds with no index
// arithmetic or predicates; only a row's last tile is predicated (padding
// slots are never added).  Symmetric: the D_Dl1 .* y scaling of a row is
// applied when the backward sweep reaches it (the same product, before any
// use).  y lives in shared memory ([row][lane], stride 33).
template <typename T, typename IO, int SWEEP, int E, int STAGES, int NACC>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    l1gs_packed_rows_kernel(const __grid_constant__ CUtensorMap tmL, const __grid_constant__ CUtensorMap tmU,
                            const PackedParams p) {
    constexpr int S = 33;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    unsigned char* wbase = smem + (size_t)warp * p.warp_bytes;
    T* ys = reinterpret_cast<T*>(wbase + p.ring_bytes + 8 * STAGES);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);
    const int ps = p.ps;

    const int wpb = blockDim.x >> 5;
    const int32_t g0 = p.gbeg + blockIdx.x * wpb + warp, gstride = gridDim.x * wpb;
    RowRing<T, E, STAGES, SWEEP> ring;
    ring.tmL = &tmL;
    ring.tmU = &tmU;
    ring.buf = reinterpret_cast<T*>(wbase);
    ring.bars = reinterpret_cast<uint64_t*>(wbase + p.ring_bytes);
    ring.gstride = gstride;
    ring.ntiles = p.ntiles;
    ring.lane = lane;
    const int32_t my_groups = g0 < p.ngroups ? (p.ngroups - 1 - g0) / gstride + 1 : 0;
    ring.total = my_groups * ((SWEEP == 2) ? 2 * p.ntiles : p.ntiles);
    ring.prologue(g0);

    int32_t c = 0;
    for (int32_t gi = 0; gi < my_groups; ++gi) {
        const int64_t g = g0 + (int64_t)gi * gstride;
        const int64_t rowbase = g * 32 * (int64_t)ps;
        T* yk = ys + lane;
        {   // x -> ys[li][partition], coalesced; (partition, li) advanced without division (ps >= 32)
            int pp = 0, li = lane;
            for (int t = lane; t < 32 * ps; t += 32) {
                const int64_t row = rowbase + t;
                ys[li * S + pp] = row < p.n ? (T)x[row] : T(0);
                li += 32;
                if (li >= ps) {
                    li -= ps;
                    ++pp;
                }
            }
        }
        __syncwarp();

        if (SWEEP != 1) {   // forward, rows ascending: slots D, a[li][0..li-1]
            int32_t t = c;
            for (int li = 0; li < ps; ++li) {
                const int len = li + 1;
                const int nt = (len + E - 1) / E;
                RowAcc<T, NACC> acc;
                if (!ring.wait(t)) goto timeout;
                const T* tl = ring.tile(t) + lane;
                const T d = tl[0];
                if (nt == 1) {
#pragma unroll
                    for (int m = 1; m < E; ++m)
                        if (m < len) acc.add(m, mul_rn(tl[m * 32], yk[(m - 1) * S]));
                } else {
                    T a[7], b[7];
#pragma unroll
                    for (int m = 1; m < 8; ++m) {
                        a[m - 1] = lds_t(tl + m * 32);
                        b[m - 1] = lds_t(yk + (m - 1) * S);
                    }
#pragma unroll
                    for (int m = 0; m < 7; ++m) acc.add(m + 1, mul_rn(a[m], b[m]));
#pragma unroll
                    for (int m0 = 8; m0 < E; m0 += 8) fold8<T, S>(acc, tl + m0 * 32, yk + (m0 - 1) * S);
                }
                ring.release(t);
                ++t;
                for (int tr = 1; tr < nt; ++tr) {
                    if (!ring.wait(t)) goto timeout;
                    tl = ring.tile(t) + lane;
                    const T* yy = yk + (tr * E - 1) * S;
                    if (tr + 1 < nt || (len & (E - 1)) == 0) {
#pragma unroll
                        for (int m0 = 0; m0 < E; m0 += 8) fold8<T, S>(acc, tl + m0 * 32, yy + m0 * S);
                    } else {
                        const int cnt = len & (E - 1);
#pragma unroll
                        for (int m = 0; m < E; ++m)
                            if (m < cnt) acc.add(m, mul_rn(tl[m * 32], yy[m * S]));
                    }
                    ring.release(t);
                    ++t;
                }
                yk[li * S] = div_rn(sub_rn(yk[li * S], acc.total()), d);
            }
            c += p.ntiles;
        }
        if (SWEEP != 0) {   // backward, rows descending: slots D, a[li][li+1..ps-1]
            int32_t t = c;
            for (int q = 0; q < ps; ++q) {
                const int li = ps - 1 - q;
                const int len = q + 1;
                const int nt = (len + E - 1) / E;
                RowAcc<T, NACC> acc;
                if (!ring.wait(t)) goto timeout;
                const T* tl = ring.tile(t) + lane;
                const T d = tl[0];
                const T* yy0 = yk + li * S;   // term slot m reads y[li + m]
                if (nt == 1) {
#pragma unroll
                    for (int m = 1; m < E; ++m)
                        if (m < len) acc.add(m, mul_rn(tl[m * 32], yy0[m * S]));
                } else {
                    T a[7], b[7];
#pragma unroll
                    for (int m = 1; m < 8; ++m) {
                        a[m - 1] = lds_t(tl + m * 32);
                        b[m - 1] = lds_t(yy0 + m * S);
                    }
#pragma unroll
                    for (int m = 0; m < 7; ++m) acc.add(m + 1, mul_rn(a[m], b[m]));
#pragma unroll
                    for (int m0 = 8; m0 < E; m0 += 8) fold8<T, S>(acc, tl + m0 * 32, yy0 + m0 * S);
                }
                ring.release(t);
                ++t;
                for (int tr = 1; tr < nt; ++tr) {
                    if (!ring.wait(t)) goto timeout;
                    tl = ring.tile(t) + lane;
                    const T* yy = yy0 + (tr * E) * S;
                    if (tr + 1 < nt || (len & (E - 1)) == 0) {
#pragma unroll
                        for (int m0 = 0; m0 < E; m0 += 8) fold8<T, S>(acc, tl + m0 * 32, yy + m0 * S);
                    } else {
                        const int cnt = len & (E - 1);
#pragma unroll
                        for (int m = 0; m < E; ++m)
                            if (m < cnt) acc.add(m, mul_rn(tl[m * 32], yy[m * S]));
                    }
                    ring.release(t);
                    ++t;
                }
                const T yi = (SWEEP == 2) ? mul_rn(d, yk[li * S]) : yk[li * S];   // y .= D_Dl1 .* y (:897)
                yk[li * S] = div_rn(sub_rn(yi, acc.total()), d);
            }
            c += p.ntiles;
        }
        __syncwarp();
        {
            int pp = 0, li = lane;
            for (int t = lane; t < 32 * ps; t += 32) {
                const int64_t row = rowbase + t;
                if (row < p.n) y[row] = (IO)ys[li * S + pp];
                li += 32;
                if (li >= ps) {
                    li -= ps;
                    ++pp;
                }
            }
        }
        __syncwarp();
    }
    return;
timeout:
    ring.drain(p.err);
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
    int32_t n, ps, kbeg, nparts;   // partitions [kbeg, nparts) of this launch
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
    for (int64_t k = p.kbeg + (int64_t)blockIdx.x * wpb + warp; k < p.nparts; k += (int64_t)gridDim.x * wpb) {
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

// View apply, thread per partition: warp per 32 consecutive partitions (the
// packed kernel's mapping).  The warp first gathers every row's in-block
// strict-lower / strict-upper entries into per-partition lists in shared
// memory, laid out [entry][lane] so each lane's reads are conflict-free and in
// the reference's order (rows ascending, columns ascending within a row); then
// each lane runs the serial row recurrence of its own partition.
constexpr int kViewStage = 256;   // entries of one 32-row step staged in shared memory

struct ViewLanesParams {
    int32_t n, ps, nparts, gbeg, ngroups;   // groups [gbeg, ngroups) of this launch
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
__global__ void __launch_bounds__(kWarpsPerBlock * 32) l1gs_view_lanes_kernel(const ViewLanesParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int S = 33;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int ps = p.ps;
    const bool want_lo = SWEEP != 1, want_up = SWEEP != 0;
    unsigned char* w = smem + (size_t)warp * p.warp_bytes;
    T* ys = reinterpret_cast<T*>(w);
    T* lval = ys + ps * S;
    T* uval = lval + p.cap_lo * 32;
    uint16_t* loff = reinterpret_cast<uint16_t*>(uval + p.cap_up * 32);
    uint16_t* uoff = loff + (ps + 1) * 32;
    uint16_t* lcol = uoff + (ps + 1) * 32;
    uint16_t* ucol = lcol + p.cap_lo * 32;
    int32_t* cntl = reinterpret_cast<int32_t*>(
        (reinterpret_cast<uintptr_t>(ucol + p.cap_up * 32) + 3) & ~uintptr_t(3));   // running list counts
    int32_t* cntu = cntl + 32;
    int32_t* sci = cntu + 32;   // one step's entries (kViewStage)
    T* sv = reinterpret_cast<T*>((reinterpret_cast<uintptr_t>(sci + kViewStage) + 7) & ~uintptr_t(7));
    const int32_t* __restrict__ rp = p.rp;
    const int32_t* __restrict__ ci = p.ci;
    const T* __restrict__ v = static_cast<const T*>(p.v);
    const T* __restrict__ D = static_cast<const T*>(p.D);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);

    const int wpb = blockDim.x >> 5;
    for (int64_t g = p.gbeg + (int64_t)blockIdx.x * wpb + warp; g < p.ngroups; g += (int64_t)gridDim.x * wpb) {
        const int64_t rowbase = g * 32 * (int64_t)ps;
        // List building, 32 consecutive rows at a time (one per lane): each
        // lane loads its row's entries (8 at a time, all in flight) once,
        // in-block entries get list slots from a segmented warp scan (the
        // lanes of one partition are contiguous), and are written in row
        // order, storage order within a row -- the reference's order.
        if (lane < 32) {
            cntl[lane] = 0;
            cntu[lane] = 0;
        }
        __syncwarp();
        // Row pointers of steps m, m+1, m+2 in registers (lane l: row
        // rowbase + 32 m + l; rows past n clamp to rp[n]), loaded three steps ahead.
        auto rp_of = [&](int m) -> int32_t { return __ldg(rp + min(rowbase + 32 * m + lane, (int64_t)p.n)); };
        int32_t r0 = rp_of(0), r1 = rp_of(1), r2 = rp_of(2);
        // Step m handles rows rowbase + 32 m + lane.  Its entries are the
        // contiguous range [qs, qe) of its first and the next step's first row
        // pointer; they are loaded coalesced (lane e takes entries e, e + 32, ...)
        // one step ahead into registers and dropped into the warp's staging
        // buffer, from which every lane then scans its own row.  A step with
        // more than kViewStage entries reads its rows from global memory instead
        // (same order).
        int32_t pc[kViewStage / 32];
        T pv[kViewStage / 32];
        T px = T(0);
        auto fetch = [&](int m, int32_t qs, int32_t qe) {
            if (m >= ps) return;
            const int32_t cnt = qe - qs;
            if (cnt <= kViewStage) {
#pragma unroll
                for (int k = 0; k < kViewStage / 32; ++k) {
                    const int32_t e = k * 32 + lane;
                    if (e < cnt) {
                        pc[k] = __ldg(ci + qs + e);
                        pv[k] = __ldg(v + qs + e);
                    }
                }
            }
            const int64_t i = rowbase + 32 * m + lane;
            if (i < p.n) px = (T)x[i];
        };
        fetch(0, __shfl_sync(0xffffffffu, r0, 0), __shfl_sync(0xffffffffu, r1, 0));
        int pp = lane / ps, li = lane - (lane / ps) * ps;
        for (int m = 0; m < ps; ++m) {
            const int64_t i = rowbase + 32 * m + lane;
            const bool valid = i < p.n;
            const int32_t r3 = rp_of(m + 3);
            const int32_t qs = __shfl_sync(0xffffffffu, r0, 0), qe = __shfl_sync(0xffffffffu, r1, 0);
            const int32_t cnt = qe - qs;
            const bool staged = cnt <= kViewStage;
            if (staged) {
#pragma unroll
                for (int k = 0; k < kViewStage / 32; ++k) {
                    const int32_t e = k * 32 + lane;
                    if (e < cnt) {
                        sci[e] = pc[k];
                        sv[e] = pv[k];
                    }
                }
            }
            ys[li * S + pp] = valid ? px : T(0);
            __syncwarp();
            fetch(m + 1, qe, __shfl_sync(0xffffffffu, r2, 0));   // in flight while this step is processed
            const int64_t s0 = rowbase + (int64_t)pp * ps;
            const int64_t e0 = min(s0 + ps - 1, (int64_t)p.n - 1);
            int32_t q1 = __shfl_down_sync(0xffffffffu, r0, 1);
            if (lane == 31) q1 = qe;
            int32_t q0 = r0;
            if (!valid) q0 = q1 = 0;
            // entries q of this step at cb[q - qo] / vb[q - qo]: the staging, or global memory
            const int32_t* cb = staged ? sci : ci;
            const T* vb = staged ? sv : v;
            const int32_t qo = staged ? qs : 0;
            const int32_t ii = (int32_t)i, si = (int32_t)s0, ei = (int32_t)e0;
            const int len = q1 - q0;
            // phase A: in-block entries as bitmasks over the row's entries (rows of
            // up to 32 entries), counted by popc; longer rows are counted in a loop
            uint32_t mlo = 0, mup = 0;
            int cl = 0, cu = 0;
            if (len <= 32) {
                for (int b = 0; b < len; ++b) {
                    const int32_t j = cb[q0 - qo + b];
                    mlo |= (uint32_t)(want_lo && j >= si && j < ii) << b;
                    mup |= (uint32_t)(want_up && j > ii && j <= ei) << b;
                }
                cl = __popc(mlo);
                cu = __popc(mup);
            } else {
                for (int32_t q = q0; q < q1; ++q) {
                    const int32_t j = cb[q - qo];
                    cl += (want_lo && j >= si && j < ii);
                    cu += (want_up && j > ii && j <= ei);
                }
            }
            // phase B: slots = running count of the partition + exclusive prefix over its lanes
            const unsigned seg = __match_any_sync(0xffffffffu, pp);
            const int first = __ffs(seg) - 1, last = 31 - __clz(seg);
            int il = cl, iu = cu;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int tl = __shfl_up_sync(0xffffffffu, il, o);
                const int tu = __shfl_up_sync(0xffffffffu, iu, o);
                if (lane >= o) {
                    il += tl;
                    iu += tu;
                }
            }
            const int basel = __shfl_sync(0xffffffffu, il - cl, first);
            const int baseu = __shfl_sync(0xffffffffu, iu - cu, first);
            int wl = cntl[pp] + (il - cl) - basel;
            int wu = cntu[pp] + (iu - cu) - baseu;
            loff[li * 32 + pp] = (uint16_t)wl;
            uoff[li * 32 + pp] = (uint16_t)wu;
            __syncwarp();
            if (lane == last) {
                cntl[pp] += il - basel;
                cntu[pp] += iu - baseu;
            }
            // phase C: write the in-block entries in storage order (set bits ascending)
            if (len <= 32) {
                while (mlo) {
                    const int b = __ffs(mlo) - 1;
                    mlo &= mlo - 1;
                    lval[wl * 32 + pp] = vb[q0 - qo + b];
                    lcol[wl * 32 + pp] = (uint16_t)(cb[q0 - qo + b] - si);
                    ++wl;
                }
                while (mup) {
                    const int b = __ffs(mup) - 1;
                    mup &= mup - 1;
                    uval[wu * 32 + pp] = vb[q0 - qo + b];
                    ucol[wu * 32 + pp] = (uint16_t)(cb[q0 - qo + b] - si);
                    ++wu;
                }
            } else {
                for (int32_t q = q0; q < q1; ++q) {
                    const int32_t j = cb[q - qo];
                    if (want_lo && j >= si && j < ii) {
                        lval[wl * 32 + pp] = vb[q - qo];
                        lcol[wl * 32 + pp] = (uint16_t)(j - si);
                        ++wl;
                    } else if (want_up && j > ii && j <= ei) {
                        uval[wu * 32 + pp] = vb[q - qo];
                        ucol[wu * 32 + pp] = (uint16_t)(j - si);
                        ++wu;
                    }
                }
            }
            __syncwarp();   // staging and counts are rewritten by the next step
            r0 = r1;
            r1 = r2;
            r2 = r3;
            li += 32;
            while (li >= ps) {
                li -= ps;
                ++pp;
            }
        }
        __syncwarp();
        loff[ps * 32 + lane] = (uint16_t)cntl[lane];
        uoff[ps * 32 + lane] = (uint16_t)cntu[lane];
        __syncwarp();
        // serial recurrence per lane (partition g*32 + lane)
        const int64_t k = g * 32 + lane;
        const int aps = k < p.nparts ? (int)min((int64_t)ps, (int64_t)p.n - k * ps) : 0;
        T* yk = ys + lane;
        const T* dk = D + k * ps;   // this lane's D_Dl1, loaded two rows ahead of use
        if (want_lo) {
            int qa = loff[lane];
            T d1 = aps > 0 ? __ldg(dk) : T(1), d2 = aps > 1 ? __ldg(dk + 1) : T(1);
            for (int li = 0; li < aps; ++li) {
                const T d = d1;
                d1 = d2;
                if (li + 2 < aps) d2 = __ldg(dk + li + 2);
                T acc = T(0);
                const int qb = loff[(li + 1) * 32 + lane];
                for (int q = qa; q < qb; ++q)
                    acc = add_rn(acc, mul_rn(lval[q * 32 + lane], yk[lcol[q * 32 + lane] * S]));
                qa = qb;
                yk[li * S] = div_rn(sub_rn(yk[li * S], acc), d);
            }
        }
        if (want_up) {   // symmetric: D_Dl1 .* y applied to a row when this sweep reaches it
            int qb = aps > 0 ? uoff[aps * 32 + lane] : 0;
            T d1 = aps > 0 ? __ldg(dk + aps - 1) : T(1), d2 = aps > 1 ? __ldg(dk + aps - 2) : T(1);
            for (int li = aps - 1; li >= 0; --li) {
                const T d = d1;
                d1 = d2;
                if (li >= 2) d2 = __ldg(dk + li - 2);
                T yi = yk[li * S];
                if (SWEEP == 2) yi = mul_rn(d, yi);
                T acc = T(0);
                const int qa = uoff[li * 32 + lane];
                for (int q = qa; q < qb; ++q)
                    acc = add_rn(acc, mul_rn(uval[q * 32 + lane], yk[ucol[q * 32 + lane] * S]));
                qb = qa;
                yk[li * S] = div_rn(sub_rn(yi, acc), d);
            }
        }
        __syncwarp();
        {
            int pp = lane / ps, li = lane - (lane / ps) * ps;
            for (int t = lane; t < 32 * ps; t += 32) {
                const int64_t i = rowbase + t;
                if (i < p.n) y[i] = (IO)ys[li * S + pp];
                li += 32;
                while (li >= ps) {
                    li -= ps;
                    ++pp;
                }
            }
        }
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
    int64_t tstore = 0;      // stream slots per direction (tlen, or rows_off(ps) in the rows layout)
    int32_t rows_layout = 0; // packed partsize >= 32: tile width of the row-aligned streams (0: classic)
    // Threads per partition of the packed sweep: 1 (thread per partition,
    // interleaved or rows layout) or 4/8/16/32 (cooperative kernel, coop layout).
    int32_t tpp = 1;
    // Partial sums per row of the thread-per-partition rows kernel: 1 (the
    // reference's order) or 4 (reordered; options.order == 2).
    int32_t nacc = 1;
    int32_t order = 1;           // 1: reference summation order everywhere; 2: reordered where faster
    int32_t coop_m = 0;          // rows per lane of the cooperative kernel
    int32_t coop_ngroups = 0;    // groups of G = 32/tpp partitions
    hscoop::Layout coop;
    hscoop::Geometry coop_geo;
    void* SC = nullptr;          // cooperative streams (all directions)
    hscoop::LaunchCache coop_lc;
    // Matrix-view cache up to partsize 128: per-group segment lists of the
    // in-block entries (the row-wise arrays are released after the build).
    hsseg::View seg;
    bool use_seg = false;
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
    // host-buffer apply: streams (copy in, copy out, then 4 apply streams) and
    // chunk events, made on first use
    cudaStream_t hstream[2 + 4] = {};
    std::vector<cudaEvent_t> hev;
    int64_t bytes = 0;
    int E = 8, stages = 4, minb = 3;
    int launch_key = -1, launch_grid = 1;
    int32_t rng_beg = 0, rng_end = -1;   // groups of the next launch (rng_end < 0: all)
    int32_t io_groups = 0, io_group_parts = 32;   // the groups rng_beg/rng_end count
    const void* launch_kernel = nullptr;
    int32_t* err_word = nullptr;
    cudaStream_t alloc_stream = nullptr;   // set: buffers are stream-ordered (cudaMallocAsync)
    bool stream_ordered = false;
};

namespace {

template <typename T>
int dmalloc(hs_l1gs* P, T** p, size_t bytes) {
    cudaError_t e = P->stream_ordered ? cudaMallocAsync((void**)p, bytes ? bytes : 1, P->alloc_stream)
                                      : cudaMalloc((void**)p, bytes ? bytes : 1);
    if (e != cudaSuccess) return hs::cuda_error(e, "cudaMalloc");
    P->bytes += (int64_t)bytes;
    return HS_OK;
}

void release(hs_l1gs* P, cudaStream_t free_stream = nullptr) {
    if (!P) return;
    for (cudaEvent_t e : P->hev) cudaEventDestroy(e);
    for (cudaStream_t q : P->hstream)
        if (q) cudaStreamDestroy(q);
    hsseg::destroy(&P->seg);
    void* ptrs[] = {P->D, P->Di, P->SLi, P->SUi, P->SC, P->rp, P->ci, P->vs, P->dev_x, P->dev_y};
    for (void* q : ptrs)
        if (q) {
            if (P->stream_ordered)
                cudaFreeAsync(q, free_stream ? free_stream : P->alloc_stream);
            else
                cudaFree(q);
        }
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

// Largest in-block strict-lower (caps[0]) and strict-upper (caps[1]) entry
// count of any partition, from device row-wise arrays (the view kernels size
// their shared-memory lists by it).  Thread per partition.
__global__ void view_caps_kernel(int32_t n, int32_t ps, int32_t nparts, const int32_t* __restrict__ rp,
                                 const int32_t* __restrict__ ci, int32_t* __restrict__ caps) {
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nparts; k += gridDim.x * blockDim.x) {
        const int64_t s = (int64_t)k * ps, e = min(s + ps - 1, (int64_t)n - 1);
        int32_t cl = 0, cu = 0;
        for (int64_t i = s; i <= e; ++i)
            for (int32_t q = rp[i]; q < rp[i + 1]; ++q) {
                const int64_t j = ci[q];
                cl += (j >= s && j < i);
                cu += (j > i && j <= e);
            }
        atomicMax(caps, cl);
        atomicMax(caps + 1, cu);
    }
}

// Where setup_device finds the row-wise arrays.
enum class Rows {
    Host,            // host memory: uploaded here, released after setup (packed) or kept (view)
    DeviceBorrowed,  // device memory owned by the caller, read during setup only (packed caches)
    DeviceOwned      // device memory allocated for this handle (P->bytes counts it): kept or freed like Host
};

template <typename TM, typename TS>
int setup_device(hs_l1gs* P, const int32_t* rp_h, const int32_t* ci_h, const TM* v_h, int64_t nnz,
                 cudaStream_t st, Rows where = Rows::Host) {
    const int32_t n = P->n;
    int32_t *rp_d = nullptr, *ci_d = nullptr;
    TM* v_d = nullptr;
    int rc;
    const bool on_device = where == Rows::DeviceBorrowed;
    if (where != Rows::Host) {
        rp_d = const_cast<int32_t*>(rp_h);
        ci_d = const_cast<int32_t*>(ci_h);
        v_d = const_cast<TM*>(v_h);
        if (where == Rows::DeviceOwned) {
            P->rp = rp_d;
            P->ci = ci_d;
        }
    } else {
        if ((rc = dmalloc(P, &rp_d, sizeof(int32_t) * (n + 1)))) return rc;
        P->rp = rp_d;
        if ((rc = dmalloc(P, &ci_d, sizeof(int32_t) * nnz))) return rc;
        P->ci = ci_d;
        if ((rc = dmalloc(P, &v_d, sizeof(TM) * nnz))) return rc;
        P->vs = v_d;   // the handle owns it from here (kept, converted or released below)
        HS_CUDA(cudaMemcpyAsync(rp_d, rp_h, sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, st));
        HS_CUDA(cudaMemcpyAsync(ci_d, ci_h, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
        HS_CUDA(cudaMemcpyAsync(v_d, v_h, sizeof(TM) * nnz, cudaMemcpyHostToDevice, st));
    }

    TS* D = nullptr;
    if ((rc = dmalloc(P, &D, sizeof(TS) * n))) return rc;
    P->D = D;
    TS *Di = nullptr, *SLi = nullptr, *SUi = nullptr;
    const bool packed = P->cache == HS_CACHE_PACKED;
    const bool lower = P->sweep != HS_SWEEP_BACKWARD, upper = P->sweep != HS_SWEEP_FORWARD;
    TS* SC = nullptr;
    if (packed && P->tpp > 1) {
        const int64_t count = (int64_t)P->coop_ngroups * P->coop.Lgp;
        if ((rc = dmalloc(P, &SC, sizeof(TS) * count))) return rc;
        P->SC = SC;
        HS_CUDA(cudaMemsetAsync(SC, 0, sizeof(TS) * count, st));
    } else if (packed) {
        if (!P->rows_layout) {   // the rows layout carries D_Dl1 inside its streams
            const int64_t dcount = (int64_t)P->ps * P->npad;
            if ((rc = dmalloc(P, &Di, sizeof(TS) * dcount))) return rc;
            P->Di = Di;
            fill_kernel<TS><<<std::min<int64_t>((dcount + 255) / 256, 4096), 256, 0, st>>>(Di, dcount, TS(1));
            HS_LAUNCH_CHECK("fill_kernel");
        }
        const int64_t tcount = P->tstore * P->npad;
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
    const int coop_dirs = (lower ? 1 : 0) | (upper ? 2 : 0);
    setup_rows_kernel<TM, TS><<<(n + 255) / 256, 256, 0, st>>>(n, P->ps, P->npad, rp_d, ci_d, v_d, (TM)P->eta, D,
                                                              Di, SLi, SUi, P->rows_layout, P->coop, coop_dirs, SC);
    HS_LAUNCH_CHECK("setup_rows_kernel");
    if (packed && P->rows_layout) {
        const int32_t lps = (int32_t)((int64_t)n - (int64_t)(P->nparts - 1) * P->ps);
        if (lps < P->ps) {
            rows_tail_kernel<TS><<<1, 256, 0, st>>>(P->ps, lps, P->npad, P->nparts - 1, P->rows_layout, SLi, SUi);
            HS_LAUNCH_CHECK("rows_tail_kernel");
        }
    }
    if (packed && on_device) {
        if (!P->stream_ordered) HS_CUDA(cudaStreamSynchronize(st));
    } else if (packed) {
        HS_CUDA(cudaStreamSynchronize(st));
        cudaFree(rp_d);
        cudaFree(ci_d);
        cudaFree(v_d);
        P->bytes -= (int64_t)(sizeof(int32_t) * (n + 1 + nnz) + sizeof(TM) * nnz);
        P->rp = nullptr;
        P->ci = nullptr;
        P->vs = nullptr;
    } else if (P->ps <= hsseg::kMaxPartsize) {
        // segment lists from the rows; the apply needs nothing else of the matrix
        if ((rc = hsseg::build<TM, TS>(n, P->ps, P->nparts, rp_d, ci_d, v_d, lower, upper, &P->seg, st))) return rc;
        P->bytes += P->seg.bytes;
        P->use_seg = true;
        P->io_groups = P->seg.ngroups;   // groups of seg.G partitions
        P->io_group_parts = P->seg.G;
        HS_CUDA(cudaStreamSynchronize(st));
        if (!on_device) {
            cudaFree(rp_d);
            cudaFree(ci_d);
            cudaFree(v_d);
            P->bytes -= (int64_t)(sizeof(int32_t) * (n + 1 + nnz) + sizeof(TM) * nnz);
        }
        P->rp = nullptr;
        P->ci = nullptr;
        P->vs = nullptr;
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
        if (where == Rows::Host) {
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
        } else {
            int32_t* caps = nullptr;
            HS_CUDA(cudaMalloc(&caps, 2 * sizeof(int32_t)));
            cudaMemsetAsync(caps, 0, 2 * sizeof(int32_t), st);
            view_caps_kernel<<<std::max(1, std::min((P->nparts + 255) / 256, 4096)), 256, 0, st>>>(
                n, P->ps, P->nparts, P->rp, P->ci, caps);
            int32_t hc[2] = {0, 0};
            cudaError_t e1 = cudaGetLastError();
            if (e1 == cudaSuccess) e1 = cudaMemcpyAsync(hc, caps, sizeof(hc), cudaMemcpyDeviceToHost, st);
            if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(st);
            cudaFree(caps);
            if (e1 != cudaSuccess) return hs::cuda_error(e1, "view_caps_kernel");
            hs::count_launch();
            ml = hc[0];
            mu = hc[1];
        }
        const int32_t limit = 4096;
        P->cap_lo = lower ? std::min(ml, limit) : 0;
        P->cap_up = upper ? std::min(mu, limit) : 0;
    }
    HS_CUDA(cudaStreamSynchronize(st));
    return HS_OK;
}

// Ring depth of the rows kernel.  A warp serves 32 partitions and keeps its
// y slice (ps x 33 values) and its ring in shared memory, so the depth sets
// how many warps fit on an SM; large partsizes have few partitions, so pick
// the depth that needs the fewest rounds of warps over the groups, then the
// deepest ring among those.
inline int rows_stages(int ps, int E, size_t es, int64_t ngroups) {
    const int cand8[] = {4, 8, 16}, cand32[] = {4, 8};
    const int* cand = E == 32 ? cand32 : cand8;
    const int ncand = E == 32 ? 2 : 3;
    const int64_t sms = hs::num_sms();
    int best = cand[0];
    int64_t best_rounds = INT64_MAX;
    for (int c = 0; c < ncand; ++c) {
        const int64_t wb = ((int64_t)E * 32 * es * cand[c] + 8 * cand[c] + (int64_t)ps * 33 * es + 127) / 128 * 128;
        const int64_t wpb = std::max<int64_t>(1, std::min<int64_t>(kWarpsPerBlock, (200 * 1024) / wb));
        const int64_t per_sm = 233472 / (wpb * wb + 1024);
        if (per_sm < 1) continue;
        const int64_t rounds = (ngroups + sms * per_sm * wpb - 1) / (sms * per_sm * wpb);
        // Fewest rounds first.  On a tie, a single round (every group resident
        // at once) takes the deeper ring, more bytes in flight per warp; several
        // rounds keep the shallower ring and its extra resident warps (at 128^3
        // partsize 32: 4 stages, 12 warps per SM, beat 8 stages, 8 warps).
        if (rounds < best_rounds || (rounds == best_rounds && rounds == 1)) {
            best_rounds = rounds;
            best = cand[c];
        }
    }
    return best;
}

// Tile geometry of the packed stream: E rows x 32 lanes per TMA tile, STAGES
// tiles in the per-warp ring.  Large partsizes keep fewer warps per SM (the
// y slice lives in shared memory), so they get bigger tiles and a deeper ring.
inline void pick_tile(int ps, int sdt, int* E, int* stages, int* minb) {
    const bool big = ps >= 128;
    if (sdt == HS_F64) { *E = big ? 16 : 8; }
    else { *E = big ? 32 : 16; }
    *stages = big ? 8 : 4;
    *minb = 3;
    // Tuning override: HSB200_L1GS_TILE="big,minb" selects the large-tile ring
    // (1) or the small one (0), and the blocks-per-SM register cap of the
    // partsize-16 kernel (3 or 4).
    if (const char* env = getenv("HSB200_L1GS_TILE")) {
        int b = -1, mb = -1;
        if (sscanf(env, "%d,%d", &b, &mb) >= 1) {
            if (b == 0 || b == 1) {
                *E = sdt == HS_F64 ? (b ? 16 : 8) : (b ? 32 : 16);
                *stages = b ? 8 : 4;
            }
            if (mb == 3 || mb == 4) *minb = mb;
        }
    }
}


template <typename KERN>
int launch_packed_kernel(KERN kern, hs_l1gs* P, PackedParams& p, int stages, bool balanced, uint32_t extra_bytes,
                         cudaStream_t st) {
    // per warp: the tile ring, one mbarrier per stage, then the kernel's slice
    p.warp_bytes = (p.ring_bytes + 8 * stages + extra_bytes + 127) / 128 * 128;
    const int wpb = (int)std::max<int64_t>(1, std::min<int64_t>(kWarpsPerBlock, (200 * 1024) / p.warp_bytes));
    const size_t smem = (size_t)p.warp_bytes * wpb;
    // The launch shape depends only on the handle and the io type: compute it once.
    const int key = (int)sizeof(p) ^ (int)p.warp_bytes ^ (wpb << 20);
    if (P->launch_key != key || P->launch_kernel != (const void*)kern) {
        int rc = hs::ensure_dynamic_smem((const void*)kern, (int)smem);
        if (rc) return rc;
        int per_sm = 0;
        HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpb * 32, smem));
        if (per_sm < 1) return hs::set_error(HS_ERR_UNSUPPORTED, "partsize %d needs too much shared memory", P->ps);
        // Every warp streams whole groups.  Balanced: size the grid so all
        // warps get the same number of groups (the fewest rounds the resident
        // warps allow) instead of a last round that only some warps run -- the
        // better shape when the stream is bandwidth-bound (FP64 coefficients).
        // Otherwise one block per resident slot: FP32 streams move half the
        // bytes per instruction and gain more from the extra warps in flight.
        if (const char* env = getenv("HSB200_GRID_FULL"))   // tuning override: 1 = full, 0 = balanced
            balanced = atoi(env) != 1;
        const int64_t slots = (int64_t)per_sm * hs::num_sms() * wpb;
        const int64_t rounds = std::max<int64_t>(1, (P->ngroups + slots - 1) / slots);
        const int64_t grid = balanced ? (P->ngroups + rounds * wpb - 1) / (rounds * wpb)
                                      : (P->ngroups + wpb - 1) / wpb;
        P->launch_grid = (int)std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)per_sm * hs::num_sms()));
        P->launch_key = key;
        P->launch_kernel = (const void*)kern;
    }
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>(P->launch_grid, ((int64_t)p.ngroups - p.gbeg + wpb - 1) / wpb));
    kern<<<grid, wpb * 32, smem, st>>>(P->tmL, P->tmU, p);
    HS_LAUNCH_CHECK("l1gs_packed_kernel");
    return HS_OK;
}

template <typename T, typename IO, int SWEEP, int E, int STAGES>
int launch_packed_t(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    PackedParams p;
    p.n = P->n;
    p.ps = P->ps;
    p.nparts = P->nparts;
    p.npad = P->npad;
    p.gbeg = P->rng_beg;
    p.ngroups = P->rng_end < 0 ? P->ngroups : P->rng_end;
    p.tlen = (int32_t)P->tlen;
    p.ntiles = (int32_t)((P->tlen + E - 1) / E);
    p.Di = P->Di;
    p.x = x;
    p.y = y;
    if (!P->err_word) P->err_word = hs::device_error_word();
    p.err = P->err_word;
    p.ring_bytes = (uint32_t)(E * 32 * sizeof(T) * STAGES);
    // Balanced grids for FP64 streams, and for FP32 streams from partsize 24
    // (measured at 128^3: 5.5 against 5.1 TB/s there; at partsizes 12 and 16
    // the full grid is 4 and 10 % faster).
#define HS_SMALL(PSV, MB)                                                                                \
    {                                                                                                    \
        constexpr int XS = (PSV % 2 == 0) ? PSV + 1 : PSV;                                               \
        return launch_packed_kernel(l1gs_packed_small_kernel<T, IO, SWEEP, PSV, E, STAGES, MB>, P, p,    \
                                    STAGES, sizeof(T) == 8 || PSV >= 24, (uint32_t)(32 * XS * sizeof(T)), \
                                    st);                                                                 \
    }
    if constexpr (STAGES == 4) {
        switch (P->ps) {
            case 2: HS_SMALL(2, 4)
            case 4: HS_SMALL(4, 4)
            case 8: HS_SMALL(8, 4)
            case 12: HS_SMALL(12, 4)
            case 16:
                if (P->minb == 4) HS_SMALL(16, 4)
                HS_SMALL(16, 3)
            case 24: HS_SMALL(24, 3)
            case 31: HS_SMALL(31, 3)
            case 32: HS_SMALL(32, 3)
            default: break;
        }
    }
#undef HS_SMALL
    return launch_packed_kernel(l1gs_packed_kernel<T, IO, SWEEP, E, STAGES>, P, p, STAGES, sizeof(T) == 8,
                                (uint32_t)(P->ps * 33 * sizeof(T)), st);
}

// Row-aligned streams (partsize >= 32): E-slot tiles (8 or 32), a ring of STAGES.
template <typename T, typename IO, int SWEEP, int E, int STAGES, int NACC>
int launch_rows_stages(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    PackedParams p;
    p.n = P->n;
    p.ps = P->ps;
    p.nparts = P->nparts;
    p.npad = P->npad;
    p.gbeg = P->rng_beg;
    p.ngroups = P->rng_end < 0 ? P->ngroups : P->rng_end;
    p.tlen = (int32_t)P->tstore;
    p.ntiles = (int32_t)(P->tstore / E);
    p.Di = nullptr;
    p.x = x;
    p.y = y;
    if (!P->err_word) P->err_word = hs::device_error_word();
    p.err = P->err_word;
    p.ring_bytes = (uint32_t)(E * 32 * sizeof(T) * STAGES);
    return launch_packed_kernel(l1gs_packed_rows_kernel<T, IO, SWEEP, E, STAGES, NACC>, P, p, STAGES, sizeof(T) == 8,
                                (uint32_t)(P->ps * 33 * sizeof(T)), st);
}

template <typename T, typename IO, int SWEEP, int NACC>
int launch_rows_n(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    if (P->rows_layout == 32) {
        if (P->stages == 4) return launch_rows_stages<T, IO, SWEEP, 32, 4, NACC>(P, x, y, st);
        return launch_rows_stages<T, IO, SWEEP, 32, 8, NACC>(P, x, y, st);
    }
    if (P->stages == 4) return launch_rows_stages<T, IO, SWEEP, 8, 4, NACC>(P, x, y, st);
    if (P->stages == 16) return launch_rows_stages<T, IO, SWEEP, 8, 16, NACC>(P, x, y, st);
    return launch_rows_stages<T, IO, SWEEP, 8, 8, NACC>(P, x, y, st);
}

template <typename T, typename IO, int SWEEP>
int launch_rows_t(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    if (P->nacc == 4) return launch_rows_n<T, IO, SWEEP, 4>(P, x, y, st);
    return launch_rows_n<T, IO, SWEEP, 1>(P, x, y, st);
}

template <typename T, typename IO, int SWEEP>
int launch_packed_cfg(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    if (P->rows_layout) return launch_rows_t<T, IO, SWEEP>(P, x, y, st);
    constexpr int EA = sizeof(T) == 8 ? 8 : 16;
    constexpr int EB = sizeof(T) == 8 ? 16 : 32;
    if (P->E == EA && P->stages == 4) return launch_packed_t<T, IO, SWEEP, EA, 4>(P, x, y, st);
    return launch_packed_t<T, IO, SWEEP, EB, 8>(P, x, y, st);
}

template <typename T, typename IO, int SWEEP>
int launch_view_lanes(hs_l1gs* P, const void* x, void* y, cudaStream_t st, size_t warp_bytes) {
    ViewLanesParams p;
    p.n = P->n;
    p.ps = P->ps;
    p.nparts = P->nparts;
    p.gbeg = P->rng_beg;
    p.ngroups = P->rng_end < 0 ? P->ngroups : P->rng_end;
    p.rp = P->rp;
    p.ci = P->ci;
    p.v = P->vs;
    p.D = P->D;
    p.x = x;
    p.y = y;
    p.cap_lo = P->cap_lo;
    p.cap_up = P->cap_up;
    p.warp_bytes = (uint32_t)warp_bytes;
    auto kern = l1gs_view_lanes_kernel<T, IO, SWEEP>;
    if (P->launch_kernel != (const void*)kern) {
        // Warps per block: the choice that keeps the most warps resident (the
        // per-block shared-memory reservation makes small blocks pay off when a
        // warp's slice is large).
        const int max_smem = (int)std::min<size_t>((size_t)kWarpsPerBlock * warp_bytes, 227 * 1024);
        if (int rc = hs::ensure_dynamic_smem((const void*)kern, max_smem)) return rc;
        int best_wpb = 0, best_warps = 0, best_per_sm = 0;
        for (int w = kWarpsPerBlock; w >= 1; w >>= 1) {
            if ((size_t)w * warp_bytes > (size_t)max_smem) continue;
            int per_sm = 0;
            HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, w * 32, (size_t)w * warp_bytes));
            if (per_sm * w > best_warps) {
                best_warps = per_sm * w;
                best_wpb = w;
                best_per_sm = per_sm;
            }
        }
        if (best_warps < 1) return hs::set_error(HS_ERR_UNSUPPORTED, "view partition needs too much shared memory");
        const int64_t want = (P->ngroups + best_wpb - 1) / best_wpb;
        P->launch_grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)best_per_sm * hs::num_sms()));
        P->launch_key = best_wpb;
        P->launch_kernel = (const void*)kern;
    }
    const int wpb = P->launch_key;
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>(P->launch_grid, ((int64_t)p.ngroups - p.gbeg + wpb - 1) / wpb));
    kern<<<grid, wpb * 32, (size_t)wpb * warp_bytes, st>>>(p);
    HS_LAUNCH_CHECK("l1gs_view_lanes_kernel");
    return HS_OK;
}

template <typename T, typename IO, int SWEEP>
int launch_view_t(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    {
        const size_t ps = (size_t)P->ps;
        const size_t lanes_bytes = (sizeof(T) * (ps * 33 + 32 * (size_t)(P->cap_lo + P->cap_up)) +
                                    sizeof(uint16_t) * (2 * (ps + 1) * 32 + 32 * (size_t)(P->cap_lo + P->cap_up)) +
                                    4 + 2 * 32 * sizeof(int32_t) + (sizeof(int32_t) + sizeof(T)) * kViewStage + 8 +
                                    127) / 128 * 128;
        if (lanes_bytes <= 100 * 1024 && P->cap_lo < 65535 && P->cap_up < 65535)
            return launch_view_lanes<T, IO, SWEEP>(P, x, y, st, lanes_bytes);
    }
    ViewParams p;
    p.n = P->n;
    p.ps = P->ps;
    p.kbeg = P->rng_beg * 32;
    p.nparts = P->rng_end < 0 ? P->nparts : std::min<int32_t>(P->nparts, P->rng_end * 32);
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
    if (int rc = hs::ensure_dynamic_smem((const void*)kern, (int)smem)) return rc;
    int per_sm = 0;
    HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpb * 32, smem));
    if (per_sm < 1) return hs::set_error(HS_ERR_UNSUPPORTED, "view partition needs too much shared memory");
    const int64_t want = ((int64_t)p.nparts - p.kbeg + wpb - 1) / wpb;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)per_sm * hs::num_sms()));
    kern<<<grid, wpb * 32, smem, st>>>(p);
    HS_LAUNCH_CHECK("l1gs_view_kernel");
    return HS_OK;
}

int launch_coop(hs_l1gs* P, const void* x, void* y, int io, cudaStream_t st) {
    hscoop::Params p;
    p.n = P->n;
    p.ps = P->ps;
    p.blk = P->coop.blk;
    p.gbeg = P->rng_beg;
    p.gend = P->rng_end < 0 ? P->coop_ngroups : P->rng_end;
    p.Lg = (int32_t)P->coop.Lg;
    p.Lgp = P->coop.Lgp;
    p.geo = P->coop_geo;
    p.SC = P->SC;
    p.D = P->D;
    p.x = x;
    p.y = y;
    if (!P->err_word) P->err_word = hs::device_error_word();
    p.err = P->err_word;
    return hscoop::launch(P->sdt, io, P->sweep, P->tpp, P->coop_m, p, &P->coop_lc, st);
}

template <typename T, typename IO>
int launch_apply(hs_l1gs* P, const void* x, void* y, cudaStream_t st) {
    if (P->cache == HS_CACHE_PACKED && P->tpp > 1) return launch_coop(P, x, y, dtype_of<IO>::value, st);
    if (P->cache == HS_CACHE_VIEW && P->use_seg) {
        if (!P->err_word) P->err_word = hs::device_error_word();
        return hsseg::launch(P->sdt, dtype_of<IO>::value, P->sweep, P->seg, P->n, P->ps, P->rng_beg,
                             P->rng_end < 0 ? P->seg.ngroups : P->rng_end, P->D, x, y, P->err_word, st);
    }
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
                for (int64_t lj = 0; lj < li; ++lj) {
                    if (P->tpp > 1) {
                        out[boff + li * (li - 1) / 2 + lj] = inter[hscoop::lower_idx(P->coop, k, li, lj)];
                        continue;
                    }
                    const int64_t e = P->rows_layout ? rows_off(li, P->rows_layout) + 1 + lj : lo_idx(li, lj);
                    out[boff + li * (li - 1) / 2 + lj] = inter[e * P->npad + k];
                }
            } else {
                const int64_t row_start = li * aps - li * (li + 1) / 2;
                for (int64_t lj = li + 1; lj < aps; ++lj) {
                    if (P->tpp > 1) {
                        out[boff + row_start + (lj - li) - 1] = inter[hscoop::upper_idx(P->coop, k, li, lj)];
                        continue;
                    }
                    const int64_t e =
                        P->rows_layout ? rows_off(ps - 1 - li, P->rows_layout) + (lj - li) : up_idx(ps, li, lj);
                    out[boff + row_start + (lj - li) - 1] = inter[e * P->npad + k];
                }
            }
        }
    }
}

}  // namespace

namespace hs {
int l1gs_view_of(const hs_l1gs* P, L1gsView* v) {
    v->n = P->n;
    v->ps = P->ps;
    v->ngroups = P->ngroups;
    v->tlen = (int32_t)P->tlen;
    v->npad = P->npad;
    v->Di = P->Di;
    v->SLi = P->SLi;
    v->SUi = P->SUi;
    v->sdt = P->sdt;
    v->sweep = P->sweep;
    v->cache = P->cache;
    return HS_OK;
}
}  // namespace hs

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace {
// Threads per partition when the caller leaves it open (0).  Partsizes from
// 30 take the blocked kernel (8 lanes per partition, off-diagonal 8 x 8 tiles
// as dense products) when padding the partition to a multiple of 8 adds at
// most 15 % to its triangle (every partsize from 32 but a few just above a
// multiple of 8 below 100, e.g. 33-37, 41-44).  Otherwise one thread per
// partition (the reference's order) while the partitions give every SM about
// six warps of 32 partitions; below that (large partsizes, small matrices)
// the column-block kernel's lanes share a partition, eight rows per lane
// where the partsize allows it.  Other partsizes below 32 keep one thread per
// partition (y and D_Dl1 of the partition in registers).
int auto_threads_per_part(int32_t ps, int64_t nparts) {
    if (ps >= 30 && hscoop::blk_padding(ps) <= 1.15) return hscoop::kBlkB;   // 30 and 31 pad to 32
    if (ps < 32) return 1;
    if (nparts / 32 >= 6 * (int64_t)hs::num_sms()) return 1;
    int tpp = 4;
    while (tpp < 32 && tpp * 8 < ps) tpp *= 2;
    const int m = hscoop::rows_per_lane(ps, tpp);
    if (m && hscoop::supported(ps, tpp, m)) return tpp;
    tpp = ps <= 128 ? 16 : 32;   // partsizes that are not lanes x rows
    const int m2 = hscoop::rows_per_lane(ps, tpp);
    return (m2 && hscoop::supported(ps, tpp, m2)) ? tpp : 1;
}

int l1gs_create_impl(const hs_sparse* A, bool on_device, int32_t partsize, int32_t is_sym, double eta, int32_t sweep,
                     int32_t cache, int32_t smoother_dtype, int32_t threads, int32_t blocks, void* stream,
                     hs_l1gs** out, bool stream_ordered = false, bool classic_small = false,
                     int32_t threads_per_part = 0, int32_t order = 0) {
    if (!out) return hs::set_error(HS_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (partsize <= 0) return hs::set_error(HS_ERR_ARG, "partsize must be greater than 0");
    if (threads <= 0) return hs::set_error(HS_ERR_ARG, "`threads` must be greater than 0");
    if (blocks <= 0) return hs::set_error(HS_ERR_ARG, "`blocks` must be greater than 0");
    if (sweep < 0 || sweep > 2) return hs::set_error(HS_ERR_ARG, "unknown sweep %d", sweep);
    if (cache != HS_CACHE_PACKED && cache != HS_CACHE_VIEW) return hs::set_error(HS_ERR_ARG, "unknown cache %d", cache);
    if (smoother_dtype != HS_F64 && smoother_dtype != HS_F32)
        return hs::set_error(HS_ERR_ARG, "unknown smoother dtype %d", smoother_dtype);
    int rc = on_device ? HS_OK : validate_sparse(A);
    if (rc) return rc;
    if (on_device && (cache != HS_CACHE_PACKED || (A->format == HS_CSC && !is_sym)))
        return hs::set_error(HS_ERR_UNSUPPORTED, "device-resident input needs a packed cache and row-wise arrays");
    if (A->dtype == HS_F32 && smoother_dtype == HS_F64)
        return hs::set_error(HS_ERR_UNSUPPORTED, "an FP64 smoother needs an FP64 matrix");
    if (partsize > 65535) return hs::set_error(HS_ERR_UNSUPPORTED, "partsize above 65535");
    if (order < 0 || order > 2) return hs::set_error(HS_ERR_ARG, "order must be 0, 1 or 2 (got %d)", order);
    if (order == 1 && threads_per_part > 1 &&
        !(sweep == HS_SWEEP_FORWARD && cache == HS_CACHE_PACKED && hscoop::blk_ok(partsize, threads_per_part)))
        return hs::set_error(HS_ERR_ARG,
                             "the reference summation order needs one thread per partition (or, for forward "
                             "sweeps, 8 lanes per partition and a partsize that is a multiple of 8)");
    if (threads_per_part != 0 && threads_per_part != 1 && threads_per_part != 4 && threads_per_part != 8 &&
        threads_per_part != 16 && threads_per_part != 32)
        return hs::set_error(HS_ERR_ARG, "threads per partition must be 0 (automatic), 1, 4, 8, 16 or 32 (got %d)",
                             threads_per_part);

    hs_l1gs* P = new hs_l1gs();
    P->stream_ordered = stream_ordered;
    P->alloc_stream = static_cast<cudaStream_t>(stream);
    P->n = A->n;
    P->ps = partsize;
    P->nparts = (int32_t)(((int64_t)A->n + partsize - 1) / partsize);
    P->npad = ((int64_t)P->nparts + 31) / 32 * 32;
    P->ngroups = (int32_t)(P->npad / 32);
    P->tlen = (int64_t)partsize * (partsize - 1) / 2;
    // Row-aligned streams for partsize >= 32: 8-slot tiles up to 96 (little
    // padding), 32-slot tiles beyond (per-tile overhead spread over 32 slots).
    // (At 32 the register-resident kernel holds 64 FP64 values of y and D_Dl1
    // per lane and spills; y in shared memory is faster.)
    // classic_small: the batch engine's kernel reads the classic layout up to 32.
    // (The rows kernel needs partsize >= 32: its x staging starts lane l at row
    // l of the group's first partition.)
    P->rows_layout =
        (cache == HS_CACHE_PACKED && partsize >= (classic_small ? 33 : 32)) ? (partsize <= 96 ? 8 : 32) : 0;
    P->tstore = P->rows_layout ? rows_off(partsize, P->rows_layout) : P->tlen;
    {   // threads per partition of the packed sweep
        int tpp = threads_per_part;
        const bool coop_ok = cache == HS_CACHE_PACKED && !classic_small && partsize >= 2;
        if (!coop_ok) {
            tpp = 1;
        } else if (tpp == 0) {
            tpp = auto_threads_per_part(partsize, P->nparts);
        }
        // The reference's summation order: one thread per partition, or the
        // blocked kernel's forward sweep (it adds in that order too).
        if (order == 1 && tpp > 1 && !(sweep == HS_SWEEP_FORWARD && hscoop::blk_ok(partsize, tpp))) tpp = 1;
        if (tpp > 1) {
            const bool blk = hscoop::blk_ok(partsize, tpp);
            const int m = blk ? partsize / tpp : hscoop::rows_per_lane(partsize, tpp);
            if (!blk && (!m || !hscoop::supported(partsize, tpp, m))) {
                if (threads_per_part != 0) {
                    delete P;
                    return hs::set_error(HS_ERR_UNSUPPORTED, "partsize %d with %d threads per partition is not provided",
                                         partsize, tpp);
                }
                tpp = 1;
            } else {
                const size_t es = dsize(smoother_dtype);
                P->tpp = tpp;
                P->coop_m = m;
                P->rows_layout = 0;
                P->tstore = 0;
                P->coop = hscoop::make_layout(partsize, tpp, sweep != HS_SWEEP_BACKWARD, sweep != HS_SWEEP_FORWARD, es);
                P->coop_ngroups = (int32_t)(((int64_t)P->nparts + P->coop.G - 1) / P->coop.G);
                P->coop_geo = hscoop::make_geometry(P->coop, es);
                if (P->coop.Lg > INT32_MAX / 2) {
                    delete P;
                    return hs::set_error(HS_ERR_UNSUPPORTED, "partsize %d is too large for %d threads per partition",
                                         partsize, tpp);
                }
            }
        }
        P->tpp = tpp;
    }
    // Summation order: reordered partial sums only when asked for (order 2)
    // and only in the rows kernel (thread per partition, partsize >= 32).
    const bool exact_order = P->tpp == 1 || (P->coop.blk && sweep == HS_SWEEP_FORWARD);
    P->order = (order == 2 || (order == 0 && !exact_order)) ? 2 : 1;
    P->nacc = (P->order == 2 && P->tpp == 1 && P->rows_layout) ? 4 : 1;
    // Host-chunked applies cut the work into whole groups of this many partitions.
    P->io_groups = P->tpp > 1 ? P->coop_ngroups : P->ngroups;
    P->io_group_parts = P->tpp > 1 ? P->coop.G : 32;
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
    // after DiagonalIndices validated the diagonal (:619, :422-436).  The
    // non-symmetric CSC is uploaded as it is; DiagonalIndices and the
    // transpose to rows run on the device.
    const int32_t* rp_h = A->ptr;
    const int32_t* ci_h = A->idx;
    const void* v_h = A->val;
    Rows where = on_device ? Rows::DeviceBorrowed : Rows::Host;
    if (A->format == HS_CSC && !is_sym) {
        int32_t *rp_d = nullptr, *ci_d = nullptr, *dg = nullptr;
        void* v_d = nullptr;
        const size_t mes = dsize(A->dtype);
        if ((rc = dmalloc(P, &rp_d, sizeof(int32_t) * ((size_t)A->n + 1))) ||
            (rc = dmalloc(P, &ci_d, sizeof(int32_t) * (size_t)A->nnz)) ||
            (rc = dmalloc(P, (char**)&v_d, mes * (size_t)A->nnz)) ||
            (rc = dmalloc(P, &dg, sizeof(int32_t) * ((size_t)A->n + 1)))) {
            cudaFree(rp_d);
            cudaFree(ci_d);
            cudaFree(v_d);
            cudaFree(dg);
            delete P;
            return rc;
        }
        P->rp = rp_d;   // released with the handle on every path below
        P->ci = ci_d;
        P->vs = v_d;
        int32_t* bad = dg + A->n;
        int32_t nb = A->n, first_bad = 0;
        cudaError_t e = cudaMemcpyAsync(bad, &nb, sizeof(int32_t), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) rc = hs::csr_from_host(A, A->dtype, rp_d, ci_d, v_d, st, dg, bad);
        else rc = hs::cuda_error(e, "DiagonalIndices");
        if (!rc) {
            P->diag.resize(A->n);
            e = cudaMemcpyAsync(&first_bad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(P->diag.data(), dg, sizeof(int32_t) * A->n, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = hs::cuda_error(e, "DiagonalIndices");
        }
        cudaFree(dg);
        P->bytes -= (int64_t)(sizeof(int32_t) * ((size_t)A->n + 1));
        if (!rc && first_bad < A->n) {
            hs::set_error(HS_ERR_SINGULAR, "SingularException(%d): missing or zero diagonal", first_bad + 1);
            rc = hs::set_singular_col(first_bad + 1);
        }
        if (rc) {
            release(P);
            return rc;
        }
        rp_h = rp_d;   // setup_device keeps the arrays (view cache) or releases them (packed)
        ci_h = ci_d;
        v_h = v_d;
        where = Rows::DeviceOwned;
    }

    if (A->dtype == HS_F64 && smoother_dtype == HS_F64)
        rc = setup_device<double, double>(P, rp_h, ci_h, static_cast<const double*>(v_h), A->nnz, st, where);
    else if (A->dtype == HS_F64)
        rc = setup_device<double, float>(P, rp_h, ci_h, static_cast<const double*>(v_h), A->nnz, st, where);
    else
        rc = setup_device<float, float>(P, rp_h, ci_h, static_cast<const float*>(v_h), A->nnz, st, where);
    if (rc) {
        release(P);
        return rc;
    }
    if (cache == HS_CACHE_PACKED && P->tpp > 1) {
        std::memset(&P->tmL, 0, sizeof(CUtensorMap));
        std::memset(&P->tmU, 0, sizeof(CUtensorMap));
    } else if (cache == HS_CACHE_PACKED) {
        pick_tile(partsize, smoother_dtype, &P->E, &P->stages, &P->minb);
        if (P->rows_layout) {   // one tile per row segment
            P->E = P->rows_layout;
            P->stages = rows_stages(P->ps, P->E, dsize(smoother_dtype), P->ngroups);
            // Tuning override: HSB200_ROWS_STAGES = tiles in flight per warp
            // (4 or 8 with 32-slot tiles, 4, 8 or 16 with 8-slot tiles).
            if (const char* env = getenv("HSB200_ROWS_STAGES")) {
                const int st = atoi(env);
                if (st == 4 || st == 8 || (P->E == 8 && st == 16)) P->stages = st;
            }
        }
        const uint32_t E = (uint32_t)P->E;
        const void* l = P->SLi ? P->SLi : P->SUi;
        const void* u = P->SUi ? P->SUi : P->SLi;
        if (l) {
            const size_t es = dsize(smoother_dtype);
            if ((rc = hs::encode_tensor_map_2d(&P->tmL, l, smoother_dtype, P->npad, P->tstore, P->npad * es, 32, E)) ||
                (rc = hs::encode_tensor_map_2d(&P->tmU, u, smoother_dtype, P->npad, P->tstore, P->npad * es, 32, E))) {
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
}  // namespace

namespace hs {
int l1gs_create_from_matrix(const hs_matrix* M, int32_t partsize, double eta, int32_t sweep, int32_t smoother_dtype,
                            cudaStream_t st, hs_l1gs** out) {
    hs_sparse d{};
    const void* v = nullptr;
    int dt = 0;
    matrix_arrays(M, &d.ptr, &d.idx, &v, &dt);
    d.n = matrix_n(M);
    d.nnz = matrix_nnz(M);
    d.format = HS_CSR;
    d.dtype = dt;
    d.val = v;
    return l1gs_create_impl(&d, true, partsize, 1, eta, sweep, HS_CACHE_PACKED, smoother_dtype, 256, 148, st, out,
                            true, /*classic_small=*/true);
}

void l1gs_destroy_async(hs_l1gs* P, cudaStream_t st) { release(P, st); }
}  // namespace hs

extern "C" {

int hs_l1gs_create(const hs_sparse* A, int32_t partsize, int32_t is_sym, double eta, int32_t sweep, int32_t cache,
                   int32_t smoother_dtype, int32_t threads, int32_t blocks, void* stream, hs_l1gs** out) {
    return l1gs_create_impl(A, false, partsize, is_sym, eta, sweep, cache, smoother_dtype, threads, blocks, stream, out);
}

int hs_l1gs_create_opts(const hs_sparse* A, int32_t partsize, int32_t is_sym, double eta, int32_t sweep,
                        int32_t cache, int32_t smoother_dtype, int32_t threads, int32_t blocks,
                        const hs_l1gs_options* opts, void* stream, hs_l1gs** out) {
    return l1gs_create_impl(A, false, partsize, is_sym, eta, sweep, cache, smoother_dtype, threads, blocks, stream, out,
                            false, false, opts ? opts->threads_per_part : 0, opts ? opts->order : 0);
}

int hs_l1gs_apply(hs_l1gs* P, const void* x, void* y, int32_t io_dtype, void* stream) {
    if (!P || !x || !y) return hs::set_error(HS_ERR_ARG, "hs_l1gs_apply: NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (P->sdt == HS_F64 && io_dtype == HS_F64) return launch_apply<double, double>(P, x, y, st);
    if (P->sdt == HS_F32 && io_dtype == HS_F32) return launch_apply<float, float>(P, x, y, st);
    if (P->sdt == HS_F32 && io_dtype == HS_F64) return launch_apply<float, double>(P, x, y, st);
    return hs::set_error(HS_ERR_UNSUPPORTED, "FP64 smoother with FP32 vectors is not provided");
}

// Host-buffer apply.  Page-locked (mapped) host vectors are read and written
// by the apply kernel itself over PCIe: every row of x is read once and every
// row of y written once, so both link directions stream concurrently with no
// staging copies.  Other host memory goes through device copies: partitions
// are independent (each reads only its own rows of x), so the groups are cut
// into chunks whose host->device copy, apply and device->host copy run on
// separate streams -- chunk c's apply waits only for chunk c's rows of x, and
// its rows of y leave as soon as it ends.
namespace {
constexpr int kHostChunks = 16;
constexpr int kHostWork = 4;                          // apply streams: chunk c on c % kHostWork
constexpr size_t kHostChunkMin = size_t(4) << 20;   // bytes of x per chunk, at least
// events: [0] fork, [1, 1+K) copy-in done, [1+K, 1+2K) apply done, [1+2K] copy-out done,
// [2+2K, 2+2K+W) apply streams done
constexpr int kEvIn = 1, kEvApply = 1 + kHostChunks, kEvOut = 1 + 2 * kHostChunks,
              kEvWork = 2 + 2 * kHostChunks, kEvCount = 2 + 2 * kHostChunks + kHostWork;

// Start of the CUDA allocation that holds address p (driver query), or 0.
uintptr_t allocation_start(const void* p) {
    using Fn = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);
    static const Fn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuPointerGetAttribute", &f, 4000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (Fn) nullptr;
        }
        return reinterpret_cast<Fn>(f);
    }();
    CUdeviceptr start = 0;
    if (!fn || fn(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, (CUdeviceptr)(uintptr_t)p) != CUDA_SUCCESS) return 0;
    return (uintptr_t)start;
}

// Device address of a page-locked, mapped host buffer of `bytes` bytes, or
// null: the first and the last byte must lie in the same mapped allocation,
// so the kernel never touches an address outside it.
void* mapped_device_pointer(const void* p, size_t bytes) {
    const char* last = static_cast<const char*>(p) + (bytes ? bytes - 1 : 0);
    cudaPointerAttributes a, b;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || cudaPointerGetAttributes(&b, last) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || b.type != cudaMemoryTypeHost || !a.devicePointer || !b.devicePointer)
        return nullptr;
    const uintptr_t s0 = allocation_start(p);
    if (!s0 || s0 != allocation_start(last)) return nullptr;
    if (static_cast<const char*>(b.devicePointer) - static_cast<const char*>(a.devicePointer) != last - static_cast<const char*>(p))
        return nullptr;
    return a.devicePointer;
}

// The chunk sequence, forked from `origin` (ev[0] recorded there) and joined
// back to it: copies in on hstream[0], chunk c's apply on work stream
// c % kHostWork after its copy in, its copy out on hstream[1] after its apply.
// Chunks touch disjoint rows, so their applies may run concurrently.
int enqueue_host_chunks(hs_l1gs* P, const void* x_host, void* y_host, void* y_mapped, int32_t io_dtype,
                        int chunks, cudaStream_t origin) {
    cudaStream_t in = P->hstream[0], out = P->hstream[1];
    cudaStream_t* work = P->hstream + 2;
    cudaEvent_t* ev = P->hev.data();
    HS_CUDA(cudaEventRecord(ev[0], origin));
    if (in != origin) HS_CUDA(cudaStreamWaitEvent(in, ev[0], 0));
    HS_CUDA(cudaStreamWaitEvent(out, ev[0], 0));
    for (int w = 0; w < kHostWork; ++w) HS_CUDA(cudaStreamWaitEvent(work[w], ev[0], 0));
    const size_t es = dsize(io_dtype);
    const int64_t rows_per_group = (int64_t)P->io_group_parts * P->ps;
    const char* xs = static_cast<const char*>(x_host);
    char* ysh = static_cast<char*>(y_host);
    char* xd = static_cast<char*>(P->dev_x);
    char* yd = static_cast<char*>(P->dev_y);
    for (int c = 0; c < chunks; ++c) {
        const int32_t gb = (int32_t)((int64_t)P->io_groups * c / chunks);
        const int32_t ge = (int32_t)((int64_t)P->io_groups * (c + 1) / chunks);
        const int64_t r0 = gb * rows_per_group, r1 = std::min<int64_t>(ge * rows_per_group, P->n);
        if (r1 <= r0) continue;
        const size_t off = es * (size_t)r0, len = es * (size_t)(r1 - r0);
        cudaStream_t wk = work[c % kHostWork];
        HS_CUDA(cudaMemcpyAsync(xd + off, xs + off, len, cudaMemcpyHostToDevice, in));
        HS_CUDA(cudaEventRecord(ev[kEvIn + c], in));
        HS_CUDA(cudaStreamWaitEvent(wk, ev[kEvIn + c], 0));
        P->rng_beg = gb;
        P->rng_end = ge;
        const int rc = hs_l1gs_apply(P, P->dev_x, y_mapped ? y_mapped : P->dev_y, io_dtype, wk);
        P->rng_beg = 0;
        P->rng_end = -1;
        if (rc) return rc;
        if (y_mapped) continue;   // the apply wrote its rows of y to the host itself
        HS_CUDA(cudaEventRecord(ev[kEvApply + c], wk));
        HS_CUDA(cudaStreamWaitEvent(out, ev[kEvApply + c], 0));
        HS_CUDA(cudaMemcpyAsync(ysh + off, yd + off, len, cudaMemcpyDeviceToHost, out));
    }
    // join: the origin resumes after every copy out and every apply stream
    HS_CUDA(cudaEventRecord(ev[kEvOut], out));
    HS_CUDA(cudaStreamWaitEvent(origin, ev[kEvOut], 0));
    for (int w = 0; w < kHostWork; ++w) {
        HS_CUDA(cudaEventRecord(ev[kEvWork + w], work[w]));
        HS_CUDA(cudaStreamWaitEvent(origin, ev[kEvWork + w], 0));
    }
    if (in != origin) {
        HS_CUDA(cudaEventRecord(ev[kEvIn + kHostChunks - 1], in));
        HS_CUDA(cudaStreamWaitEvent(origin, ev[kEvIn + kHostChunks - 1], 0));
    }
    return HS_OK;
}

}  // namespace

int hs_l1gs_apply_host(hs_l1gs* P, const void* x_host, void* y_host, int32_t io_dtype, void* stream) {
    if (!P || !x_host || !y_host) return hs::set_error(HS_ERR_ARG, "hs_l1gs_apply_host: NULL argument");
    const size_t es = dsize(io_dtype);
    const size_t bytes = es * (size_t)P->n;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // 2 (default): the apply reads x and writes y in mapped host memory; 1: x
    // through staging copies, y written straight to the host; 0: staging
    // copies both ways
    int zero_copy = 2;
    if (const char* env = getenv("HSB200_HOST_ZEROCOPY"))   // tuning override
        zero_copy = atoi(env);
    void* ym = zero_copy >= 1 ? mapped_device_pointer(y_host, bytes) : nullptr;
    if (zero_copy >= 2 && ym) {
        void* xm = mapped_device_pointer(x_host, bytes);
        if (xm) {
            const int rc = hs_l1gs_apply(P, xm, ym, io_dtype, stream);
            if (rc) return rc;
            HS_CUDA(cudaStreamSynchronize(st));
            return HS_OK;
        }
    }
    if (!P->dev_x) {
        int rc;
        if ((rc = dmalloc(P, &P->dev_x, bytes))) return rc;
        if ((rc = dmalloc(P, &P->dev_y, bytes))) return rc;
    }
    int64_t want = std::max<size_t>(1, bytes / kHostChunkMin);
    if (const char* env = getenv("HSB200_HOST_CHUNKS"))   // tuning override
        want = std::max(1, atoi(env));
    const int chunks = (int)std::min<int64_t>(std::min<int64_t>(kHostChunks, P->io_groups), want);
    if (chunks <= 1) {
        HS_CUDA(cudaMemcpyAsync(P->dev_x, x_host, bytes, cudaMemcpyHostToDevice, st));
        int rc = hs_l1gs_apply(P, P->dev_x, ym ? ym : P->dev_y, io_dtype, stream);
        if (rc) return rc;
        if (!ym) HS_CUDA(cudaMemcpyAsync(y_host, P->dev_y, bytes, cudaMemcpyDeviceToHost, st));
        HS_CUDA(cudaStreamSynchronize(st));
        return HS_OK;
    }
    if (!P->hstream[0]) {
        for (cudaStream_t& q : P->hstream) HS_CUDA(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
        P->hev.resize(kEvCount);
        for (cudaEvent_t& e : P->hev) HS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const int rc = enqueue_host_chunks(P, x_host, y_host, ym, io_dtype, chunks, st);
    const cudaError_t se = cudaStreamSynchronize(st);
    if (rc) return rc;
    if (se != cudaSuccess) return hs::cuda_error(se, "hs_l1gs_apply_host");
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
    info->threads_per_part = P->tpp;
    const bool exact = (P->tpp == 1 && P->nacc == 1) || (P->tpp > 1 && P->coop.blk && P->sweep == HS_SWEEP_FORWARD);
    info->order = exact ? 1 : 2;
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
    const void* src = P->tpp > 1 ? P->SC : (which == 0 ? P->SLi : P->SUi);
    const bool has = which == 0 ? P->sweep != HS_SWEEP_BACKWARD : P->sweep != HS_SWEEP_FORWARD;
    if (!has) return hs::set_error(HS_ERR_ARG, "this sweep has no %s buffer", which == 0 ? "SL" : "SU");
    if (capacity < P->S) return hs::set_error(HS_ERR_ARG, "capacity %lld < %lld", (long long)capacity, (long long)P->S);
    const size_t es = dsize(P->sdt);
    std::memset(out_host, 0, es * P->S);
    if (!src) return HS_OK;  // partsize 1: empty triangles
    std::vector<unsigned char> inter(P->tpp > 1 ? es * (size_t)P->coop_ngroups * P->coop.Lgp
                                                : es * P->tstore * P->npad);
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
