// The cooperative packed sweep kernel (layout and order of operations:
// l1gs_coop.cuh).  Included by one translation unit per sweep direction
// (l1gs_coop_fwd.cu, l1gs_coop_bwd.cu, l1gs_coop_sym.cu), each compiling the
// kernels of HS_COOP_SWEEP only.
#pragma once

#include <algorithm>

#include "l1gs_coop.cuh"

namespace hscoop {

constexpr int kCoopWarps = 4;   // warps per block; every warp streams its own groups

// SWEEP: 0 forward, 1 backward, 2 symmetric.  TPP lanes per partition, up to M
// rows per lane; EXACT: the partsize is exactly TPP * M (no row predicates).
// Lane 0 of each warp keeps the warp's ring filled with 1D bulk copies,
// nst - 1 chunks ahead of the sweep, across group boundaries.
template <typename T, typename IO, int SWEEP, int TPP, int M, bool EXACT>
__global__ void __launch_bounds__(kCoopWarps * 32) l1gs_coop_kernel(const Params p) {
    constexpr int G = 32 / TPP;
    constexpr unsigned FULL = 0xffffffffu;
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

    const int g = lane / TPP, r = lane % TPP;
    const int ps = EXACT ? TPP * M : p.ps;
    const int mcount = EXACT ? M : (ps + TPP - 1) / TPP;   // row slots per lane in use
    const uint32_t rmask = (che * nst) - 1u;
    const T* ring = reinterpret_cast<const T*>(wbase);
    T* ys = reinterpret_cast<T*>(wbase + geo.ys_off);   // y of row t of partition g at ys[t * G + g]
    T* ds = reinterpret_cast<T*>(wbase + geo.ds_off);   // D_Dl1, same layout
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
    // acc[m] += a * v on the rows of slot m (row r + TPP m); `act` adds the
    // partition's row predicate for partsizes that are not TPP * M.
    auto fma_slot = [&](T* acc, int m, const T* pl, int off, T v, bool act) {
        if (act && (EXACT || r + TPP * m < ps)) acc[m] = add_rn(acc[m], mul_rn(pl[off], v));
    };

    for (int32_t gi = 0; gi < my_groups; ++gi) {
        const int64_t q = q0 + (int64_t)gi * qstride;
        const int32_t c0 = gi * nchg;                  // first chunk of this group
        const uint32_t vg = (uint32_t)c0 << l2;        // ring position of the group's entry 0 (mod 2^32)
        const int64_t rowbase = q * G * (int64_t)ps;   // the group's rows are contiguous
        for (int idx = lane; idx < G * ps; idx += 32) {
            const int pp = idx / ps, t = idx - pp * ps;
            const int64_t row = rowbase + idx;
            const bool valid = row < p.n;
            ys[t * G + pp] = valid ? (T)x[row] : T(0);
            ds[t * G + pp] = valid ? D[row] : T(1);
        }
        __syncwarp();
        T acc[M];
#pragma unroll
        for (int m = 0; m < M; ++m) acc[m] = T(0);
        uint32_t lpos = 0;   // group-stream position of the current column block

        if (SWEEP != 1) {   // forward: columns j = 0 .. ps-1
            // value of row 0 (its accumulator is 0); then, per column t, the
            // value of row t+1 is computed as soon as its accumulator is final
            T vcur = div_rn(sub_rn(ys[g], T(0)), ds[g]);
#pragma unroll
            for (int mb = 0; mb < M; ++mb) {
                if (!EXACT && mb >= mcount) break;
                for (int tr = 0; tr < TPP; ++tr) {
                    const int t = mb * TPP + tr;
                    if (r == tr) ys[t * G + g] = vcur;
                    if (t >= ps - 1) break;   // the last row updates nothing
                    const uint32_t cnt = (uint32_t)(G * (ps - 1 - t));
                    const T ynx = ys[(t + 1) * G + g], dnx = ds[(t + 1) * G + g];
                    const int32_t need = c0 + (int32_t)((lpos + cnt - 1) >> l2);
                    if (need >= ready && !wait_upto(need)) {
                        ok = false;
                        break;
                    }
                    // entry of row i = r + TPP m (i > t): e = i - t - 1, at (e * G + g)
                    const T* pl = ring + ((vg + lpos) & rmask) + ((r - tr - 1) * G + g);
                    // the slots that hold row t+1 first: m = mb (rows after t) and m = mb + 1
                    fma_slot(acc, mb, pl, 0, vcur, r > tr);
                    if (mb + 1 < M) fma_slot(acc, mb + 1, pl, 32, vcur, true);
                    T an;
                    if (mb + 1 < M)
                        an = __shfl_sync(FULL, tr == TPP - 1 ? acc[mb + 1] : acc[mb], (tr + 1) & (TPP - 1), TPP);
                    else
                        an = __shfl_sync(FULL, acc[mb], (tr + 1) & (TPP - 1), TPP);
                    const T vnext = div_rn(sub_rn(ynx, an), dnx);
#pragma unroll
                    for (int m = mb + 2; m < M; ++m) {
                        if (!EXACT && m >= mcount) break;
                        fma_slot(acc, m, pl, 32 * (m - mb), vcur, true);
                    }
                    lpos += cnt;
                    const int32_t done = c0 + (int32_t)(lpos >> l2);
                    if (done > freed) release(done);
                    vcur = vnext;
                }
                if (!ok) break;
            }
        }
        if (!ok) break;
        if (SWEEP == 2) {   // y .= D_Dl1 .* y (:897); rows past n restart from 0
            __syncwarp();
            for (int idx = lane; idx < G * ps; idx += 32) {
                const int pp = idx % G, t = idx / G;
                const bool valid = rowbase + (int64_t)pp * ps + t < p.n;
                ys[idx] = valid ? mul_rn(ds[idx], ys[idx]) : T(0);
            }
            __syncwarp();
#pragma unroll
            for (int m = 0; m < M; ++m) acc[m] = T(0);
        }
        if (SWEEP != 0) {   // backward: columns j = ps-1 .. 0
            T vcur = div_rn(sub_rn(ys[(ps - 1) * G + g], T(0)), ds[(ps - 1) * G + g]);
#pragma unroll
            for (int mb = M - 1; mb >= 0; --mb) {
                if (!EXACT && mb >= mcount) continue;
                for (int tr = TPP - 1; tr >= 0; --tr) {
                    const int j = mb * TPP + tr;
                    if (!EXACT && j >= ps) continue;
                    if (r == tr) ys[j * G + g] = vcur;
                    if (j == 0) break;
                    const uint32_t cnt = (uint32_t)(G * j);
                    const T ynx = ys[(j - 1) * G + g], dnx = ds[(j - 1) * G + g];
                    const int32_t need = c0 + (int32_t)((lpos + cnt - 1) >> l2);
                    if (need >= ready && !wait_upto(need)) {
                        ok = false;
                        break;
                    }
                    // entry of row i = r + TPP m (i < j): e = i, at (e * G + g)
                    const T* pl = ring + ((vg + lpos) & rmask) + (r * G + g);
                    // the slots that hold row j-1 first: m = mb (rows before j) and m = mb - 1
                    fma_slot(acc, mb, pl, 32 * mb, vcur, r < tr);
                    if (mb >= 1) fma_slot(acc, mb - 1, pl, 32 * (mb - 1), vcur, true);
                    T an;
                    if (mb >= 1)
                        an = __shfl_sync(FULL, tr == 0 ? acc[mb - 1] : acc[mb], (tr - 1) & (TPP - 1), TPP);
                    else
                        an = __shfl_sync(FULL, acc[mb], (tr - 1) & (TPP - 1), TPP);
                    const T vnext = div_rn(sub_rn(ynx, an), dnx);
#pragma unroll
                    for (int m = 0; m + 1 < mb; ++m) fma_slot(acc, m, pl, 32 * m, vcur, true);
                    lpos += cnt;
                    const int32_t done = c0 + (int32_t)(lpos >> l2);
                    if (done > freed) release(done);
                    vcur = vnext;
                }
                if (!ok) break;
            }
        }
        if (!ok) break;
        if (c0 + nchg > freed) release(c0 + nchg);   // the group's last, partly used chunk
        __syncwarp();
        for (int idx = lane; idx < G * ps; idx += 32) {
            const int pp = idx / ps, t = idx - pp * ps;
            const int64_t row = rowbase + idx;
            if (row < p.n) y[row] = (IO)ys[t * G + pp];
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

template <typename T, typename IO, int SWEEP, int TPP, int M, bool EXACT>
int launch_t(const Params& p, LaunchCache* lc, cudaStream_t st) {
    auto kern = l1gs_coop_kernel<T, IO, SWEEP, TPP, M, EXACT>;
    if (lc->kern != (const void*)kern) {
        // Warps per block: the choice that keeps the most warps resident.
        int best_w = 0, best_warps = 0, best_per_sm = 0;
        for (int w = kCoopWarps; w >= 1; w >>= 1) {
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
    HS_LAUNCH_CHECK("l1gs_coop_kernel");
    return HS_OK;
}

// The (lanes per partition, rows per lane) pairs with kernels: every pair for
// partsizes that are exactly lanes x rows, 16 and 32 lanes for the others
// (keep in step with hscoop::supported; 8 lanes run the blocked kernel).
#define HS_COOP_EXACT_PAIRS(X) \
    X(4, 4) X(4, 8) X(4, 16) X(16, 4) X(16, 8) X(16, 16) X(32, 4) X(32, 8) X(32, 16)
#define HS_COOP_GENERIC_PAIRS(X) X(16, 4) X(16, 8) X(16, 16) X(32, 4) X(32, 8) X(32, 16)

template <typename T, typename IO, int SWEEP>
int launch_pair(int tpp, int m, bool exact, const Params& p, LaunchCache* lc, cudaStream_t st) {
#define HS_COOP_EXACT(TP, MM) \
    if (exact && tpp == TP && m == MM) return launch_t<T, IO, SWEEP, TP, MM, true>(p, lc, st);
#define HS_COOP_GENERIC(TP, MM) \
    if (!exact && tpp == TP && m == MM) return launch_t<T, IO, SWEEP, TP, MM, false>(p, lc, st);
    HS_COOP_EXACT_PAIRS(HS_COOP_EXACT)
    HS_COOP_GENERIC_PAIRS(HS_COOP_GENERIC)
#undef HS_COOP_EXACT
#undef HS_COOP_GENERIC
    return hs::set_error(HS_ERR_UNSUPPORTED, "no cooperative sweep for partsize %d with %d lanes", p.ps, tpp);
}

template <int SWEEP>
int launch_dir(int sdt, int io, int tpp, int m, const Params& p, LaunchCache* lc, cudaStream_t st) {
    const bool exact = p.ps == tpp * m;
    if (sdt == HS_F64 && io == HS_F64) return launch_pair<double, double, SWEEP>(tpp, m, exact, p, lc, st);
    if (sdt == HS_F32 && io == HS_F32) return launch_pair<float, float, SWEEP>(tpp, m, exact, p, lc, st);
    if (sdt == HS_F32 && io == HS_F64) return launch_pair<float, double, SWEEP>(tpp, m, exact, p, lc, st);
    return hs::set_error(HS_ERR_UNSUPPORTED, "FP64 smoother with FP32 vectors is not provided");
}

}  // namespace hscoop
