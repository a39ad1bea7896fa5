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
// in the reference.
//
// A warp's group stream is one contiguous run read front to back, so the
// lanes load each tile straight from global memory (16-byte loads, 512
// contiguous bytes per warp instruction), one tile ahead of the arithmetic in
// registers, while lane 0 keeps the next 16 KiB of the stream on its way into
// L2 (cp.async.bulk.prefetch.L2, no multicast).  Shared memory holds only y
// of the group.
#include "l1gs_coop.cuh"

namespace hscoop {
namespace {

constexpr int kBlkWarps = 4;   // warps per block; every warp streams its own groups
constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t kPfStep = 4096;    // bytes per L2 prefetch
constexpr uint32_t kPfAhead = 16384;  // bytes kept prefetched ahead of the reads

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

__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reinterpret_cast<uint64_t>(src)), "r"(bytes)
                 : "memory");
}

// SWEEP: 0 forward, 1 backward, 2 symmetric.
template <typename T, typename IO, int SWEEP>
__global__ void __launch_bounds__(kBlkWarps * 32, 1) l1gs_blk_kernel(const Params p) {
    constexpr int B = kBlkB, G = 32 / B, V = 16 / (int)sizeof(T), NV = B / V;
    constexpr uint32_t TILE = 32 * B;              // entries of an off-diagonal warp tile
    constexpr uint32_t DG = G * B * (B - 1) / 2;   // entries of a diagonal warp tile
    static_assert(B - 1 <= NV * V, "a diagonal tile's entries fit the item buffer");
    using VT = typename Vec<T>::type;
    using VO = Vec<T>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / B, r = lane % B;
    const int ps = p.ps, nb = ps / B;
    const int wpb = blockDim.x >> 5;
    const int32_t qstride = gridDim.x * wpb;
    const int32_t q0 = p.gbeg + blockIdx.x * wpb + warp;
    T* ys = reinterpret_cast<T*>(smem + (size_t)warp * p.geo.warp_bytes);   // y of the group, natural row order
    const T* __restrict__ SC = static_cast<const T*>(p.SC);
    const T* __restrict__ D = static_cast<const T*>(p.D);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);
    const uint32_t lg_bytes = (uint32_t)p.Lg * (uint32_t)sizeof(T);

    for (int32_t q = q0; q < p.gend; q += qstride) {
        const T* gs = SC + (int64_t)q * p.Lgp;                 // the group stream
        const int64_t rowbase = (int64_t)q * G * ps;           // the group's rows are contiguous
        const int64_t prow = rowbase + (int64_t)g * ps + r;    // this lane's row of block 0
        T* yg = ys + g * ps;                                   // this lane's partition
        uint32_t pf = 0;                                       // stream bytes requested into L2 (lane 0)
        auto prefetch_to = [&](uint32_t upto) {
            if (lane == 0) {
                while (pf < upto && pf < lg_bytes) {
                    const uint32_t nbytes = min(kPfStep, (lg_bytes - pf + 15u) & ~15u);
                    prefetch_l2(reinterpret_cast<const unsigned char*>(gs) + pf, nbytes);
                    pf += nbytes;
                }
            }
        };
        // this lane's entries of the off-diagonal tile at `pos` (columns in order)
        auto load_tile = [&](VT* buf, uint32_t pos) {
            const VT* src = reinterpret_cast<const VT*>(gs + pos) + lane;
#pragma unroll
            for (int v = 0; v < NV; ++v) buf[v] = __ldg(src + v * 32);
        };
        // this lane's entries of the diagonal tile at `pos`: slot c holds column c
        // (lower, rows below it) or column c + 1 (upper, rows above it)
        auto load_diag = [&](VT* buf, uint32_t pos, bool lower) {
            const T* dp = gs + pos;
#pragma unroll
            for (int c = 0; c < B - 1; ++c) {
                T val = T(0);
                if (lower) {
                    if (r > c) val = __ldg(dp + G * (c * (B - 1) - c * (c - 1) / 2) + g * (B - 1 - c) + (r - c - 1));
                } else {
                    const int cu = c + 1;
                    if (r < cu) val = __ldg(dp + G * (B * (B - 1) / 2 - cu * (cu + 1) / 2) + g * cu + r);
                }
                VO::set(buf[c / V], c % V, val);
            }
        };
        auto tile = [&](T acc, const VT* buf, int J) -> T {
            const VT* yp = reinterpret_cast<const VT*>(yg + J * B);
#pragma unroll
            for (int v = 0; v < NV; ++v) acc = VO::dot(acc, buf[v], yp[v]);
            return acc;
        };

        if (SWEEP != 1) {   // forward: row blocks 0 .. nb-1
            prefetch_to(kPfAhead);
            int64_t row = prow;
            T xr = row < p.n ? (T)x[row] : T(0), dr = row < p.n ? D[row] : T(1);
            VT cur[NV], nxt[NV];
            int I = 0, J = 0;   // the item: tile (I, J) while J < I, then the diagonal tile of I
            uint32_t pos = 0;
            load_diag(cur, 0, true);
            T acc = T(0);
            while (true) {
                const bool is_tile = J < I;
                const uint32_t npos = pos + (is_tile ? TILE : DG);
                const int In = is_tile ? I : I + 1;
                const int Jn = is_tile ? J + 1 : 0;
                const bool more = In < nb;
                if (more) {   // the next item's entries, one item ahead
                    if (Jn < In)
                        load_tile(nxt, npos);
                    else
                        load_diag(nxt, npos, true);
                }
                prefetch_to(npos * (uint32_t)sizeof(T) + kPfAhead);
                if (is_tile) {
                    acc = tile(acc, cur, J);
                } else {
                    T yown = T(0);
#pragma unroll
                    for (int c = 0; c < B; ++c) {
                        const T v = div_rn(sub_rn(xr, acc), dr);
                        const T yc = __shfl_sync(FULL, v, c, B);
                        if (r == c) yown = v;
                        if (c < B - 1 && r > c) acc = add_rn(acc, mul_rn(VO::get(cur[c / V], c % V), yc));
                    }
                    // rows past n (a short last partition, padding partitions) stay 0
                    yg[I * B + r] = row < p.n ? yown : T(0);
                    __syncwarp();
                    acc = T(0);
                    row += B;
                    if (more) {
                        xr = row < p.n ? (T)x[row] : T(0);
                        dr = row < p.n ? D[row] : T(1);
                    }
                }
                if (!more) break;
#pragma unroll
                for (int v = 0; v < NV; ++v) cur[v] = nxt[v];
                I = In;
                J = Jn;
                pos = npos;
            }
        }
        if (SWEEP != 0) {   // backward: row blocks nb-1 .. 0
            const uint32_t base = SWEEP == 2 ? (uint32_t)p.Lg / 2 : 0u;
            prefetch_to(base * (uint32_t)sizeof(T) + kPfAhead);
            int64_t row = prow + (int64_t)(nb - 1) * B;
            T xn = (SWEEP == 1 && row < p.n) ? (T)x[row] : T(0), dr = row < p.n ? D[row] : T(1);
            VT cur[NV], nxt[NV];
            int I = nb - 1, J = nb;   // the item: tile (I, J) while J < nb, then the diagonal tile of I
            uint32_t pos = base;
            load_diag(cur, pos, false);
            T acc = T(0);
            while (true) {
                const bool is_tile = J < nb;
                const uint32_t npos = pos + (is_tile ? TILE : DG);
                const int In = is_tile ? I : I - 1;
                const int Jn = is_tile ? J + 1 : I;   // block I-1 starts with its tile J = I
                const bool more = In >= 0;
                if (more) {
                    if (Jn < nb)
                        load_tile(nxt, npos);
                    else
                        load_diag(nxt, npos, false);
                }
                prefetch_to(npos * (uint32_t)sizeof(T) + kPfAhead);
                if (is_tile) {
                    acc = tile(acc, cur, J);
                } else {
                    // symmetric: y .= D_Dl1 .* y (:897) for the block's rows, then the backward solve
                    const T xr = SWEEP == 2 ? mul_rn(dr, yg[I * B + r]) : xn;
                    T yown = T(0);
#pragma unroll
                    for (int c = B - 1; c >= 0; --c) {
                        const T v = div_rn(sub_rn(xr, acc), dr);
                        const T yc = __shfl_sync(FULL, v, c, B);
                        if (r == c) yown = v;
                        if (c > 0 && r < c) acc = add_rn(acc, mul_rn(VO::get(cur[(c - 1) / V], (c - 1) % V), yc));
                    }
                    yg[I * B + r] = row < p.n ? yown : T(0);
                    __syncwarp();
                    acc = T(0);
                    row -= B;
                    if (more) {
                        if (SWEEP == 1) xn = row < p.n ? (T)x[row] : T(0);
                        dr = row < p.n ? D[row] : T(1);
                    }
                }
                if (!more) break;
#pragma unroll
                for (int v = 0; v < NV; ++v) cur[v] = nxt[v];
                I = In;
                J = Jn;
                pos = npos;
            }
        }
        __syncwarp();
        for (int t = lane; t < G * ps; t += 32) {
            const int64_t rr = rowbase + t;
            if (rr < p.n) y[rr] = (IO)ys[t];
        }
        __syncwarp();
    }
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
    if (p.ps % kBlkB != 0) return hs::set_error(HS_ERR_UNSUPPORTED, "blocked sweep needs a partsize that is a multiple of 8");
    if (sdt == HS_F64 && io == HS_F64) return launch_sweep<double, double>(sweep, p, lc, st);
    if (sdt == HS_F32 && io == HS_F32) return launch_sweep<float, float>(sweep, p, lc, st);
    if (sdt == HS_F32 && io == HS_F64) return launch_sweep<float, double>(sweep, p, lc, st);
    return hs::set_error(HS_ERR_UNSUPPORTED, "FP64 smoother with FP32 vectors is not provided");
}

}  // namespace hscoop
