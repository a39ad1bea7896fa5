// Blocked cooperative packed sweep: 8 lanes per partition, 4 partitions per
// warp, left-looking over 8 x 8 tiles (layout and order of operations:
// l1gs_coop.cuh, "blocked variant").
//
// Reference: the packed sweep of src/l1_gauss_seidel.jl (:1068-1095 with the
// accumulations :1547-1585): y_i = (y_i - acc_i) / D_i, acc_i the sum of
// a_ij y_j over the partition's strict triangle in ascending j.  Row block I
// of a partition first takes the off-diagonal tiles of the blocks solved
// before it: lane (g, r) adds a_{row, J*8 + c} * y_{J*8 + c} for c = 0..7, two
// or four columns per 16-byte load, y of block J read from shared memory
// (one address per partition: a broadcast).  Then the diagonal tile: at step
// c every lane forms (x - acc) / D, lane c's value is the solved y and is
// broadcast to the partition's lanes by a shuffle, and the rows after c add
// a_{row, c} * y_c.  Only the eight steps of a diagonal tile form a serial
// chain; the off-diagonal tiles, all but 8/ps of the entries, are plain
// independent multiply-adds.  Multiply and add are rounded separately, as
// in the reference.  Forward sweeps divide by D_Dl1 at every step (the
// reference's operations: bit-identical); backward and symmetric sweeps,
// which agree with the reference to rounding anyway, multiply by 1/D_Dl1
// (one division per row instead of eight).
//
// A warp walks its groups' streams item by item (an item: one off-diagonal
// warp tile, 2 KiB in FP64, or one diagonal warp tile) in the order the
// sweep uses them.  Each item is copied into a per-warp ring of kRing slots
// in shared memory by 16-byte cp.async copies of all 32 lanes, kRing - 1
// items ahead of the arithmetic; cp.async.wait_group counts the items that
// have landed, so no barrier or flag is waited on.  Shared memory holds the
// ring and y of the group.
#include "l1gs_coop.cuh"

namespace hscoop {
namespace {

constexpr int kBlkWarps = 4;   // warps per block; every warp streams its own groups
constexpr unsigned FULL = 0xffffffffu;
constexpr int kRing = 4;   // item slots per warp: kRing - 1 items in flight

template <typename T>
struct Vec;
template <>
struct Vec<double> {
    using type = double2;
    static __device__ __forceinline__ double dot(double acc, const double2& a, const double2& y) {
        acc = add_rn(acc, mul_rn(a.x, y.x));
        return add_rn(acc, mul_rn(a.y, y.y));
    }
    static __device__ __forceinline__ double get(const double2& v, int c) { return c == 0 ? v.x : v.y; }
    static __device__ __forceinline__ void set(double2& v, int c, double t) {
        if (c == 0)
            v.x = t;
        else
            v.y = t;
    }
};
template <>
struct Vec<float> {
    using type = float4;
    static __device__ __forceinline__ float dot(float acc, const float4& a, const float4& y) {
        acc = add_rn(acc, mul_rn(a.x, y.x));
        acc = add_rn(acc, mul_rn(a.y, y.y));
        acc = add_rn(acc, mul_rn(a.z, y.z));
        return add_rn(acc, mul_rn(a.w, y.w));
    }
    static __device__ __forceinline__ float get(const float4& v, int c) {
        return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
    }
    static __device__ __forceinline__ void set(float4& v, int c, float t) {
        if (c == 0)
            v.x = t;
        else if (c == 1)
            v.y = t;
        else if (c == 2)
            v.z = t;
        else
            v.w = t;
    }
};

// Position in a warp's item sequence: for each of its groups, the forward
// items (row blocks 0..nb-1: tiles J = 0..I-1, then the diagonal tile), then
// the backward items (row blocks nb-1..0: tiles J = I+1..nb-1, then the
// diagonal tile), as the sweep has them.
template <int SWEEP>
struct ItemCursor {
    int32_t q;      // group
    int32_t dir;    // 0 forward (lower stream), 1 backward (upper stream)
    int32_t I, J;   // row block; tile column block (J == I forward, J == nb backward: the diagonal tile)
    uint32_t pos;   // entry position inside the group stream
    bool valid;

    __device__ __forceinline__ void start_group(int32_t q_, int32_t gend, int nb) {
        q = q_;
        valid = q < gend;
        if (SWEEP == 1) {
            dir = 1;
            I = nb - 1;
            J = nb;
        } else {
            dir = 0;
            I = 0;
            J = 0;
        }
        pos = 0;
    }
    __device__ __forceinline__ bool is_tile(int nb) const { return dir == 0 ? J < I : J < nb; }
    __device__ __forceinline__ void advance(int nb, uint32_t Lg, int32_t qstride, int32_t gend, uint32_t tile,
                                            uint32_t dg) {
        const bool t = is_tile(nb);
        pos += t ? tile : dg;
        if (dir == 0) {
            if (t) {
                ++J;
            } else if (++I, J = 0, I == nb) {
                if (SWEEP == 2) {   // the upper stream follows in the same group
                    dir = 1;
                    I = nb - 1;
                    J = nb;
                    pos = Lg / 2;
                } else {
                    start_group(q + qstride, gend, nb);
                }
            }
        } else {
            if (t) {
                ++J;
            } else if (--I < 0) {
                start_group(q + qstride, gend, nb);
            } else {
                J = I + 1;
            }
        }
    }
};

// SWEEP: 0 forward, 1 backward, 2 symmetric.
template <typename T, typename IO, int SWEEP>
__global__ void __launch_bounds__(kBlkWarps * 32) l1gs_blk_kernel(const Params p) {
    constexpr int B = kBlkB, G = 32 / B, V = 16 / (int)sizeof(T), NV = B / V;
    constexpr uint32_t TILE = 32 * B;              // entries of an off-diagonal warp tile
    constexpr uint32_t DG = G * B * (B - 1) / 2;   // entries of a diagonal warp tile
    constexpr uint32_t SLOT = TILE;                // entries of a ring slot (the larger item)
    constexpr int CH_TILE = TILE * sizeof(T) / 16, CH_DG = DG * sizeof(T) / 16;   // 16-byte chunks
    static_assert(CH_TILE % 32 == 0, "whole copies per lane");
    using VT = typename Vec<T>::type;
    using VO = Vec<T>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / B, r = lane % B;
    const int ps = p.ps, psb = (ps + B - 1) / B * B, nb = psb / B;   // rows past ps: zero padding
    const int wpb = blockDim.x >> 5;
    const int32_t qstride = gridDim.x * wpb;
    const int32_t q0 = p.gbeg + blockIdx.x * wpb + warp;
    T* ring = reinterpret_cast<T*>(smem + (size_t)warp * p.geo.warp_bytes);   // kRing slots
    T* ys = ring + kRing * SLOT;                                              // y of the group, natural row order
    const T* __restrict__ SC = static_cast<const T*>(p.SC);
    const T* __restrict__ D = static_cast<const T*>(p.D);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);

    // Copies run kRing - 1 items ahead; one commit group per item (empty past the end).
    ItemCursor<SWEEP> ic;
    ic.start_group(q0, p.gend, nb);
    auto issue = [&](int slot) {
        if (ic.valid) {
            const int nch = ic.is_tile(nb) ? CH_TILE : CH_DG;
            const unsigned char* src = reinterpret_cast<const unsigned char*>(SC + (int64_t)ic.q * p.Lgp + ic.pos);
            unsigned char* dst = reinterpret_cast<unsigned char*>(ring + slot * SLOT);
#pragma unroll
            for (int c = 0; c < CH_TILE / 32; ++c) {
                const int k = lane + 32 * c;
                if (k < nch) hsdev::cp_async_cg16(dst + 16 * k, src + 16 * k);
            }
            ic.advance(nb, (uint32_t)p.Lg, qstride, p.gend, TILE, DG);
        }
        hsdev::cp_async_commit();
    };
#pragma unroll
    for (int s = 0; s < kRing - 1; ++s) issue(s);
    int32_t k = 0;   // items consumed
    auto next_item = [&]() -> const T* {
        hsdev::cp_async_wait<kRing - 2>();   // item k has landed (this lane's copies) ...
        __syncwarp();                        // ... and every lane's; slot (k - 1) is free
        issue((k + kRing - 1) & (kRing - 1));
        const T* slot = ring + (k & (kRing - 1)) * SLOT;
        ++k;
        return slot;
    };

    for (int32_t q = q0; q < p.gend; q += qstride) {
        const int64_t rowbase = (int64_t)q * G * ps;           // the group's rows are contiguous
        const int64_t prow = rowbase + (int64_t)g * ps + r;    // this lane's row of block 0
        T* yg = ys + g * psb;                                  // this lane's partition (padded)
        // row li of this lane's partition holds a real row: li < ps and inside the matrix
        auto real = [&](int li, int64_t row) { return li < ps && row < p.n; };
        auto tile = [&](T acc, const T* tp, int J) -> T {
            const VT* ap = reinterpret_cast<const VT*>(tp) + lane;
            const VT* yp = reinterpret_cast<const VT*>(yg + J * B);
#pragma unroll
            for (int v = 0; v < NV; ++v) acc = VO::dot(acc, ap[v * 32], yp[v]);
            return acc;
        };
        if (SWEEP != 1) {   // forward: row blocks 0 .. nb-1
            int64_t row = prow;
            T xr = real(r, row) ? (T)x[row] : T(0), dr = real(r, row) ? D[row] : T(1);
            for (int I = 0; I < nb; ++I) {
                T acc = T(0);
                for (int J = 0; J < I; ++J) acc = tile(acc, next_item(), J);
                const T* dp = next_item();
                T aj[B - 1];
#pragma unroll
                for (int c = 0; c < B - 1; ++c)
                    aj[c] = r > c ? dp[G * (c * (B - 1) - c * (c - 1) / 2) + g * (B - 1 - c) + (r - c - 1)] : T(0);
                T yown = T(0);
                // Backward and symmetric sweeps agree with the reference to rounding
                // anyway: there each lane divides once (1/D_Dl1) and the eight steps
                // multiply.  Forward sweeps divide at every step (bit-identical).
                const T rinv = SWEEP == 0 ? T(0) : div_rn(T(1), dr);
#pragma unroll
                for (int c = 0; c < B; ++c) {
                    const T v = SWEEP == 0 ? div_rn(sub_rn(xr, acc), dr) : mul_rn(sub_rn(xr, acc), rinv);
                    const T yc = __shfl_sync(FULL, v, c, B);
                    if (r == c) yown = v;
                    if (c < B - 1 && r > c) acc = add_rn(acc, mul_rn(aj[c], yc));
                }
                // rows past n (a short last partition, padding partitions) stay 0
                yg[I * B + r] = real(I * B + r, row) ? yown : T(0);
                __syncwarp();
                row += B;
                if (I + 1 < nb) {   // the next block's x and D_Dl1
                    const bool v = real((I + 1) * B + r, row);
                    xr = v ? (T)x[row] : T(0);
                    dr = v ? D[row] : T(1);
                }
            }
        }
        if (SWEEP != 0) {   // backward: row blocks nb-1 .. 0
            int64_t row = prow + (int64_t)(nb - 1) * B;
            const bool v0 = real((nb - 1) * B + r, row);
            T xn = (SWEEP == 1 && v0) ? (T)x[row] : T(0), dr = v0 ? D[row] : T(1);
            for (int I = nb - 1; I >= 0; --I) {
                T acc = T(0);
                for (int J = I + 1; J < nb; ++J) acc = tile(acc, next_item(), J);
                const T* dp = next_item();
                T au[B];
#pragma unroll
                for (int c = 1; c < B; ++c)
                    au[c] = r < c ? dp[G * (B * (B - 1) / 2 - c * (c + 1) / 2) + g * c + r] : T(0);
                // symmetric: y .= D_Dl1 .* y (:897) for the block's rows, then the backward solve
                const T xr = SWEEP == 2 ? mul_rn(dr, yg[I * B + r]) : xn;
                const T rinv = div_rn(T(1), dr);
                T yown = T(0);
#pragma unroll
                for (int c = B - 1; c >= 0; --c) {
                    const T v = mul_rn(sub_rn(xr, acc), rinv);
                    const T yc = __shfl_sync(FULL, v, c, B);
                    if (r == c) yown = v;
                    if (c > 0 && r < c) acc = add_rn(acc, mul_rn(au[c], yc));
                }
                yg[I * B + r] = real(I * B + r, row) ? yown : T(0);
                __syncwarp();
                row -= B;
                if (I > 0) {
                    const bool v = real((I - 1) * B + r, row);
                    if (SWEEP == 1) xn = v ? (T)x[row] : T(0);
                    dr = v ? D[row] : T(1);
                }
            }
        }
        for (int t = lane; t < G * psb; t += 32) {
            const int pp = t / psb, li = t - pp * psb;
            if (li >= ps) continue;
            const int64_t rr = rowbase + (int64_t)pp * ps + li;
            if (rr < p.n) y[rr] = (IO)ys[t];
        }
        __syncwarp();
    }
    hsdev::cp_async_wait<0>();   // nothing left in flight (the tail commits are empty)
}

template <typename T, typename IO, int SWEEP>
int launch_t(const Params& p, LaunchCache* lc, cudaStream_t st) {
    auto kern = l1gs_blk_kernel<T, IO, SWEEP>;
    if (lc->kern != (const void*)kern) {
        // Warps per block: the choice that keeps the most warps resident.
        int best_w = 0, best_warps = 0, best_per_sm = 0;
        for (int w = kBlkWarps; w >= 1; w >>= 1) {
            const size_t smem = (size_t)w * p.geo.warp_bytes;
            if (smem > 227 * 1024) continue;
            if (int rc = hs::ensure_dynamic_smem((const void*)kern, (int)smem)) return rc;
            int per_sm = 0;
            HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, w * 32, smem));
            if (per_sm * w > best_warps) {
                best_warps = per_sm * w;
                best_w = w;
                best_per_sm = per_sm;
            }
        }
        if (best_warps < 1) return hs::set_error(HS_ERR_UNSUPPORTED, "partsize %d needs too much shared memory", p.ps);
        lc->kern = (const void*)kern;
        lc->wpb = best_w;
        lc->per_sm = best_per_sm;
    }
    // Every warp takes the same number of groups: the fewest rounds the
    // resident warps allow, spread evenly.
    const int64_t ngr = (int64_t)p.gend - p.gbeg;
    const int64_t slots = (int64_t)lc->per_sm * hs::num_sms() * lc->wpb;
    const int64_t rounds = std::max<int64_t>(1, (ngr + slots - 1) / slots);
    const int64_t grid = std::max<int64_t>(1, (ngr + rounds * lc->wpb - 1) / (rounds * lc->wpb));
    kern<<<(int)grid, lc->wpb * 32, (size_t)lc->wpb * p.geo.warp_bytes, st>>>(p);
    HS_LAUNCH_CHECK("l1gs_blk_kernel");
    return HS_OK;
}

template <typename T, typename IO>
int launch_sweep(int sweep, const Params& p, LaunchCache* lc, cudaStream_t st) {
    switch (sweep) {
        case HS_SWEEP_FORWARD: return launch_t<T, IO, 0>(p, lc, st);
        case HS_SWEEP_BACKWARD: return launch_t<T, IO, 1>(p, lc, st);
        default: return launch_t<T, IO, 2>(p, lc, st);
    }
}

}  // namespace

int launch_blk(int sdt, int io, int sweep, const Params& p, LaunchCache* lc, cudaStream_t st) {
    if (sdt == HS_F64 && io == HS_F64) return launch_sweep<double, double>(sweep, p, lc, st);
    if (sdt == HS_F32 && io == HS_F32) return launch_sweep<float, float>(sweep, p, lc, st);
    if (sdt == HS_F32 && io == HS_F64) return launch_sweep<float, double>(sweep, p, lc, st);
    return hs::set_error(HS_ERR_UNSUPPORTED, "FP64 smoother with FP32 vectors is not provided");
}

}  // namespace hscoop
