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
// in the reference.  The streams pass through a per-warp ring of 2 KiB
// chunks filled by 1D bulk copies (cp.async.bulk, no multicast) as in the
// column-block kernel, tail stages repeating the first ones so every tile is
// one linear run.
#include "l1gs_coop.cuh"

namespace hscoop {
namespace {

constexpr int kBlkWarps = 4;   // warps per block; every warp streams its own groups
constexpr unsigned FULL = 0xffffffffu;

template <typename T>
struct Vec;
template <>
struct Vec<double> {
    using type = double2;
    static __device__ __forceinline__ double dot(double acc, const double2& a, const double2& y) {
        acc = add_rn(acc, mul_rn(a.x, y.x));
        return add_rn(acc, mul_rn(a.y, y.y));
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
};

// SWEEP: 0 forward, 1 backward, 2 symmetric.
template <typename T, typename IO, int SWEEP>
__global__ void __launch_bounds__(kBlkWarps * 32, 1) l1gs_blk_kernel(const Params p) {
    constexpr int B = kBlkB, G = 32 / B, V = 16 / (int)sizeof(T);
    constexpr uint32_t TILE = 32 * B;                 // entries of an off-diagonal warp tile
    constexpr uint32_t DG = G * B * (B - 1) / 2;      // entries of a diagonal warp tile
    using VT = typename Vec<T>::type;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Geometry geo = p.geo;
    const uint32_t l2 = geo.che_log2, che = 1u << l2, nst = geo.nst, ntail = geo.ntail;
    const int32_t nchg = (int32_t)(((uint32_t)p.Lg + che - 1) >> l2);   // chunks per group stream
    const int wpb = blockDim.x >> 5;
    const int32_t qstride = gridDim.x * wpb;
    unsigned char* wbase = smem + (size_t)warp * geo.warp_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(wbase + geo.bars_off);
    const int32_t q0 = p.gbeg + blockIdx.x * wpb + warp;
    const int32_t my_groups = q0 < p.gend ? (p.gend - 1 - q0) / qstride + 1 : 0;
    const int32_t total = my_groups * nchg;
    const T* __restrict__ SC = static_cast<const T*>(p.SC);

    // Producer state (lane 0): the next chunk to fetch and its source.
    int32_t issued = 0, pc = 0, pg = 0;
    const T* src = SC + (int64_t)q0 * p.Lgp;
    auto issue_next = [&]() {
        const uint32_t s = (uint32_t)issued & (nst - 1u);
        uint32_t bytes = che * (uint32_t)sizeof(T);
        if (pc == nchg - 1) bytes = (((uint32_t)p.Lg - ((uint32_t)pc << l2)) * (uint32_t)sizeof(T) + 15u) & ~15u;
        const bool dup = s < ntail;
        T* ringw = reinterpret_cast<T*>(wbase);
        hsdev::mbar_arrive_expect_tx(bars + s, dup ? 2 * bytes : bytes);
        hsdev::bulk_load(ringw + (size_t)s * che, src, bytes, bars + s);
        if (dup) hsdev::bulk_load(ringw + (size_t)(nst + s) * che, src, bytes, bars + s);
        ++issued;
        if (++pc == nchg) {
            pc = 0;
            ++pg;
            src = SC + ((int64_t)q0 + (int64_t)pg * qstride) * p.Lgp;
        } else {
            src += che;
        }
    };
    if (lane == 0) {
        for (uint32_t s = 0; s < nst; ++s) hsdev::mbar_init(bars + s, 1);
        hsdev::fence_barrier_init();
        while (issued < total && issued < (int32_t)nst) issue_next();
    }
    __syncwarp();

    const int g = lane / B, r = lane % B;
    const int ps = p.ps, nb = ps / B;
    const uint32_t rmask = (che * nst) - 1u;
    const T* ring = reinterpret_cast<const T*>(wbase);
    T* ys = reinterpret_cast<T*>(wbase + geo.ys_off);   // y of the group's rows, natural order ([partition][row])
    const T* __restrict__ D = static_cast<const T*>(p.D);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);

    int32_t ready = 0;   // chunks known to have landed
    int32_t freed = 0;   // chunks handed back to the producer
    bool ok = true;
    auto wait_upto = [&](int32_t last) -> bool {   // bounded
        while (ready <= last) {
            const bool got = hsdev::mbar_wait_bounded(bars + ((uint32_t)ready & (nst - 1u)),
                                                      ((uint32_t)ready / nst) & 1u);
            if (!__all_sync(FULL, got)) return false;
            ++ready;
        }
        return true;
    };
    auto release = [&](int32_t upto) {   // chunks below `upto` are consumed: refill their stages
        freed = upto;
        __syncwarp();
        if (lane == 0) {
            hsdev::fence_proxy_async_smem();
            while (issued < total && issued < freed + (int32_t)nst) issue_next();
        }
    };

    for (int32_t gi = 0; gi < my_groups && ok; ++gi) {
        const int64_t q = q0 + (int64_t)gi * qstride;
        const int32_t c0 = gi * nchg;                  // first chunk of this group
        const uint32_t vg = (uint32_t)c0 << l2;        // ring position of the group's entry 0 (mod 2^32)
        const int64_t rowbase = q * G * (int64_t)ps;   // the group's rows are contiguous
        const int64_t prow = rowbase + (int64_t)g * ps + r;   // this lane's row of block 0
        T* yg = ys + g * ps;                           // this lane's partition
        uint32_t pos = 0;                              // group-stream position
        // the run [pos, pos + len) has landed (bounded wait)
        auto have = [&](uint32_t len) -> bool {
            const int32_t need = c0 + (int32_t)((pos + len - 1) >> l2);
            return need < ready || wait_upto(need);
        };
        auto consumed = [&]() {
            const int32_t done = c0 + (int32_t)(pos >> l2);
            if (done > freed) release(done);
        };
        // sum over the off-diagonal tile at pos with y of block J
        auto tile = [&](T acc, int J) -> T {
            const T* tp = ring + ((vg + pos) & rmask) + lane * V;
            const T* yp = yg + J * B;
#pragma unroll
            for (int pv = 0; pv < B / V; ++pv)
                acc = Vec<T>::dot(acc, *reinterpret_cast<const VT*>(tp + pv * 32 * V),
                                  *reinterpret_cast<const VT*>(yp + pv * V));
            return acc;
        };

        if (SWEEP != 1) {   // forward: row blocks 0 .. nb-1
            int64_t row = prow;
            T xn = row < p.n ? (T)x[row] : T(0), dn = row < p.n ? D[row] : T(1);
            for (int I = 0; I < nb; ++I) {
                const bool valid = row < p.n;
                const T xr = xn, dr = dn;
                if (I + 1 < nb) {   // next block's x and D_Dl1, one block ahead
                    const int64_t rn = row + B;
                    xn = rn < p.n ? (T)x[rn] : T(0);
                    dn = rn < p.n ? D[rn] : T(1);
                }
                T acc = T(0);
                for (int J = 0; J < I; ++J) {
                    if (!have(TILE)) {
                        ok = false;
                        break;
                    }
                    acc = tile(acc, J);
                    pos += TILE;
                    consumed();
                }
                if (!ok) break;
                if (!have(DG)) {
                    ok = false;
                    break;
                }
                const T* dp = ring + ((vg + pos) & rmask);
                T aj[B - 1];
#pragma unroll
                for (int c = 0; c < B - 1; ++c)
                    aj[c] = r > c ? dp[G * (c * (B - 1) - c * (c - 1) / 2) + g * (B - 1 - c) + (r - c - 1)] : T(0);
                T yown = T(0);
#pragma unroll
                for (int c = 0; c < B; ++c) {
                    const T v = div_rn(sub_rn(xr, acc), dr);
                    const T yc = __shfl_sync(FULL, v, c, B);
                    if (r == c) yown = v;
                    if (c < B - 1 && r > c) acc = add_rn(acc, mul_rn(aj[c], yc));
                }
                // rows past n (a short last partition, padding partitions) stay 0
                yg[I * B + r] = valid ? yown : T(0);
                __syncwarp();
                pos += DG;
                consumed();
                row += B;
            }
        }
        if (!ok) break;
        if (SWEEP != 0) {   // backward: row blocks nb-1 .. 0
            int64_t row = prow + (int64_t)(nb - 1) * B;
            T xn = (SWEEP == 1 && row < p.n) ? (T)x[row] : T(0), dn = row < p.n ? D[row] : T(1);
            for (int I = nb - 1; I >= 0; --I) {
                const bool valid = row < p.n;
                const T dr = dn;
                // symmetric: y .= D_Dl1 .* y (:897) for the block's rows, then the backward solve
                const T xr = SWEEP == 2 ? mul_rn(dr, yg[I * B + r]) : xn;
                if (I > 0) {
                    const int64_t rn = row - B;
                    if (SWEEP == 1) xn = rn < p.n ? (T)x[rn] : T(0);
                    dn = rn < p.n ? D[rn] : T(1);
                }
                T acc = T(0);
                for (int J = I + 1; J < nb; ++J) {
                    if (!have(TILE)) {
                        ok = false;
                        break;
                    }
                    acc = tile(acc, J);
                    pos += TILE;
                    consumed();
                }
                if (!ok) break;
                if (!have(DG)) {
                    ok = false;
                    break;
                }
                const T* dp = ring + ((vg + pos) & rmask);
                T au[B];
#pragma unroll
                for (int c = 1; c < B; ++c)
                    au[c] = r < c ? dp[G * (B * (B - 1) / 2 - c * (c + 1) / 2) + g * c + r] : T(0);
                T yown = T(0);
#pragma unroll
                for (int c = B - 1; c >= 0; --c) {
                    const T v = div_rn(sub_rn(xr, acc), dr);
                    const T yc = __shfl_sync(FULL, v, c, B);
                    if (r == c) yown = v;
                    if (c > 0 && r < c) acc = add_rn(acc, mul_rn(au[c], yc));
                }
                __syncwarp();   // every lane has read yg[I * B + r] above
                yg[I * B + r] = valid ? yown : T(0);
                __syncwarp();
                pos += DG;
                consumed();
                row -= B;
            }
        }
        if (!ok) break;
        if (c0 + nchg > freed) release(c0 + nchg);   // the group's last, partly used chunk
        __syncwarp();
        for (int t = lane; t < G * ps; t += 32) {
            const int64_t rr = rowbase + t;
            if (rr < p.n) y[rr] = (IO)ys[t];
        }
        __syncwarp();
    }
    if (!ok) {
        // A bounded wait ran out: record it, let the copies in flight land
        // (bounded), and return.
        if (lane == 0) hsdev::report_error(p.err, hsdev::kErrWaitTimeout);
        const int32_t end = __shfl_sync(FULL, issued, 0);
        for (int32_t c = ready; c < end; ++c)
            (void)hsdev::mbar_wait_bounded(bars + ((uint32_t)c & (nst - 1u)), ((uint32_t)c / nst) & 1u);
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
