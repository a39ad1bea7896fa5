// Matrix-view L1 Gauss-Seidel over per-group segment lists: build and apply
// (layout and order of operations: l1gs_seg.cuh).
#include <algorithm>
#include <vector>

#include "l1gs_seg.cuh"
#include "l1gs_seg_ring.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kSegWarps = 4;

// In-block lower (s <= j < i) and upper (i < j <= e) entries of row i: their
// counts and first storage positions (contiguous: columns are sorted).
__global__ void seg_count_kernel(int32_t n, int32_t ps, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 int32_t* __restrict__ cntL, int32_t* __restrict__ qL, int32_t* __restrict__ cntU,
                                 int32_t* __restrict__ qU) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = (i / ps) * ps, e = min(s + ps - 1, (int64_t)n - 1);
        const int32_t q0 = rp[i], q1 = rp[i + 1];
        int32_t cl = 0, cu = 0, ql = q0, qu = q0;
        for (int32_t q = q0; q < q1; ++q) {
            const int64_t j = ci[q];
            if (j >= s && j < i) {
                if (cl == 0) ql = q;
                ++cl;
            } else if (j > i && j <= e) {
                if (cu == 0) qu = q;
                ++cu;
            }
        }
        cntL[i] = cl;
        qL[i] = ql;
        cntU[i] = cu;
        qU[i] = qu;
    }
}

// One warp per (group, row): the largest count of the G partitions' rows.
__global__ void seg_max_kernel(int32_t n, int32_t ps, int32_t psq, int32_t G, int32_t nparts, int64_t items,
                               const int32_t* __restrict__ cnt, uint8_t* __restrict__ maxc) {
    const int lane = threadIdx.x & 31;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < items;
         w += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t g = w / ps, li = w - g * ps;
        const int64_t k = g * G + lane, row = k * ps + li;
        const int32_t c = (lane < G && k < nparts && row < n) ? cnt[row] : 0;
        const unsigned m = __reduce_max_sync(FULL, (unsigned)c);
        if (lane == 0) maxc[g * psq + li] = (uint8_t)m;
    }
}

// Per group: the first slot of every row in the sweep's row order (ascending
// rows for the lower lists, descending for the upper), and the group's total.
__global__ void seg_off_kernel(int32_t ngroups, int32_t ps, int32_t psq, const uint8_t* __restrict__ maxc,
                               uint16_t* __restrict__ off, int32_t* __restrict__ total, int descending) {
    for (int32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x) {
        int32_t acc = 0;
        for (int32_t t = 0; t < ps; ++t) {
            const int64_t li = descending ? ps - 1 - t : t;
            off[(int64_t)g * ps + li] = (uint16_t)acc;
            acc += maxc[(int64_t)g * psq + li];
        }
        total[g] = acc;
    }
}

// Every slot's columns start as `ps` (the zero row); the scatter then writes
// the real entries over them.
template <typename TS>
__global__ void seg_pad_kernel(int64_t slots, int32_t ps, int32_t G, unsigned char* __restrict__ stream) {
    const int64_t SB = hsseg::slot_bytes(G, sizeof(TS));
    const int64_t m = slots * G;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t slot = e / G, lane = e - slot * G;
        reinterpret_cast<uint16_t*>(stream + slot * SB + G * sizeof(TS))[lane] = (uint16_t)ps;
    }
}

template <typename TM, typename TS>
__global__ void seg_scatter_kernel(int32_t n, int32_t ps, int32_t G, const int32_t* __restrict__ ci,
                                   const TM* __restrict__ v, const int32_t* __restrict__ cnt,
                                   const int32_t* __restrict__ q0, const uint16_t* __restrict__ off,
                                   const int64_t* __restrict__ base, unsigned char* __restrict__ stream) {
    const int64_t SB = hsseg::slot_bytes(G, sizeof(TS));
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / ps, li = i - k * ps, g = k / G, lane = k - g * G, s = k * ps;
        const int64_t slot0 = base[g] + off[g * ps + li];
        for (int32_t t = 0; t < cnt[i]; ++t) {
            const int32_t q = q0[i] + t;
            unsigned char* sp = stream + (slot0 + t) * SB;
            reinterpret_cast<TS*>(sp)[lane] = (TS)v[q];
            reinterpret_cast<uint16_t*>(sp + G * sizeof(TS))[lane] = (uint16_t)(ci[q] - s);
        }
    }
}

int grid_of(int64_t m) { return (int)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, 8192)); }

struct Tmp {
    std::vector<void*> p;
    ~Tmp() {
        for (void* q : p) cudaFree(q);
    }
    template <typename T>
    int get(T** out, size_t bytes) {
        cudaError_t e = cudaMalloc((void**)out, bytes ? bytes : 8);
        if (e != cudaSuccess) return hs::cuda_error(e, "cudaMalloc (segment lists)");
        p.push_back(*out);
        return HS_OK;
    }
};

template <typename T>
int dalloc(hsseg::View* view, T** out, size_t bytes) {
    cudaError_t e = cudaMalloc((void**)out, bytes ? bytes : 8);
    if (e != cudaSuccess) return hs::cuda_error(e, "cudaMalloc (segment lists)");
    view->bytes += (int64_t)bytes;
    return HS_OK;
}

// ---------------------------------------------------------------------------
// Apply: warp per group of 32 partitions, lane = partition.
// ---------------------------------------------------------------------------
using hsseg::kTab;
using hsseg::TabEnt;

// Slots per chunk: 4 (FP64, 1280 bytes) or 6 (FP32, 1152 bytes).
template <typename T>
constexpr int seg_k() {
    return sizeof(T) == 8 ? 4 : 6;
}

// Runtime partsize (2..512): y and D_Dl1 of the group in shared memory.  G
// partitions per group; lanes G..31 repeat lanes 0..G-1 (same loads, same
// values written), so no lane needs a guard.
template <typename T, typename IO, int SWEEP, int G>
__global__ void __launch_bounds__(kSegWarps * 32, 1) l1gs_seg_kernel(const hsseg::Params p) {
    constexpr int S = G + 1;
    constexpr uint32_t SB = hsseg::slot_bytes(G, sizeof(T));   // bytes per slot
    constexpr int K = seg_k<T>() * (32 / G);               // slots per chunk
    constexpr int NDIR = SWEEP == 2 ? 2 : 1;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, pl = lane & (G - 1);
    const int ps = p.ps, psq = (ps + 3) & ~3;
    unsigned char* wbase = smem + (size_t)warp * p.warp_bytes;
    T* ys = reinterpret_cast<T*>(wbase + p.ys_off);   // y of row li, partition pl: ys[li * S + pl]; row ps: +0
    T* ds = reinterpret_cast<T*>(wbase + p.ds_off);
    uint8_t* mxs = wbase + p.mx_off;                   // the group's slots per row, per direction (psq bytes each)
    const T* __restrict__ D = static_cast<const T*>(p.D);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);
    const int wpb = blockDim.x >> 5;
    hsseg::SegStream<SB, K, NDIR, SWEEP> rs;
    rs.ring = wbase + p.ring_off;
    rs.bars = reinterpret_cast<uint64_t*>(wbase + p.bars_off);
    rs.tab = reinterpret_cast<TabEnt*>(wbase + p.tab_off);
    rs.nst = p.nst;
    rs.q0 = p.gbeg + blockIdx.x * wpb + warp;
    rs.qstride = gridDim.x * wpb;
    rs.lo = p.lo;
    rs.up = p.up;
    const int32_t my_groups = rs.q0 < p.gend ? (p.gend - 1 - rs.q0) / rs.qstride + 1 : 0;
    ys[ps * S + pl] = T(0);
    rs.init(lane, my_groups);
    bool ok = true;

    // (partition, row) of this lane's t-th element of a group, t = lane + 32 u
    const int dq = 32 / ps, dr = 32 - dq * ps;
    int32_t ch = 0;   // chunk of the next slot
    for (int32_t gi = 0; gi < my_groups && ok; ++gi) {
        const int64_t g = rs.q0 + (int64_t)gi * rs.qstride;
        const int64_t rowbase = g * G * (int64_t)ps;
        const int32_t nrows = (int32_t)min((int64_t)G * ps, (int64_t)p.n - rowbase);
        // x and D_Dl1 of the group's rows -> [li][partition], all loads in flight at once
        if constexpr (sizeof(IO) == sizeof(T)) {
            int pp = lane / ps, li = lane - pp * ps;
            for (int t = lane; t < G * ps; t += 32) {
                T* yd = ys + li * S + pp;
                T* dd = ds + li * S + pp;
                if (t < nrows) {
                    hsdev::cp_async<sizeof(T)>(yd, x + rowbase + t);
                    hsdev::cp_async<sizeof(T)>(dd, D + rowbase + t);
                } else {
                    *yd = T(0);
                    *dd = T(1);
                }
                li += dr;
                pp += dq;
                if (li >= ps) {
                    li -= ps;
                    ++pp;
                }
            }
        } else {   // FP64 vectors, FP32 smoother: x converted on the way in
            int pp = lane / ps, li = lane - pp * ps;
            for (int t0 = lane; t0 < G * ps; t0 += 32 * 8) {
                IO xv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int t = t0 + 32 * u;
                    xv[u] = t < nrows ? x[rowbase + t] : IO(0);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int t = t0 + 32 * u;
                    if (t < G * ps) {
                        T* dd = ds + li * S + pp;
                        ys[li * S + pp] = (T)xv[u];
                        if (t < nrows)
                            hsdev::cp_async<sizeof(T)>(dd, D + rowbase + t);
                        else
                            *dd = T(1);
                    }
                    li += dr;
                    pp += dq;
                    if (li >= ps) {
                        li -= ps;
                        ++pp;
                    }
                }
            }
        }
        // slots per row of each direction, staged as words
#pragma unroll
        for (int d = 0; d < NDIR; ++d)
            for (int w = lane; w < psq / 4; w += 32)
                reinterpret_cast<uint32_t*>(mxs + d * psq)[w] =
                    reinterpret_cast<const uint32_t*>(rs.dir(d).maxc + g * psq)[w];
        hsdev::cp_async_wait_all();
        __syncwarp();
        T* yk = ys + pl;
        const T* dk = ds + pl;
#pragma unroll
        for (int d = 0; d < NDIR; ++d) {
            if (!ok) break;
            const bool lowerdir = SWEEP == 0 || (SWEEP == 2 && d == 0);
            const uint8_t* mx = mxs + d * psq;
            int wi = 0;   // slot of the next entry inside chunk ch
            for (int t = 0; t < ps; ++t) {
                const int li = lowerdir ? t : ps - 1 - t;
                const int m = mx[li];
                const T dv = dk[li * S];
                T yi = yk[li * S];
                T acc = T(0);
                for (int k = 0; k < m; ++k) {
                    if (ch >= rs.ready && !rs.wait_upto(ch)) {
                        ok = false;
                        break;
                    }
                    const unsigned char* sp = rs.slot(ch, wi);
                    const T a = reinterpret_cast<const T*>(sp)[pl];
                    const int col = reinterpret_cast<const uint16_t*>(sp + G * sizeof(T))[pl];
                    acc = add_rn(acc, mul_rn(a, yk[col * S]));
                    // a finished chunk goes back at once: a row may span more chunks than the ring holds
                    if (++wi == K) {
                        wi = 0;
                        ++ch;
                        rs.release(ch, lane);
                    }
                }
                if (!ok) break;
                if (SWEEP == 2 && !lowerdir) yi = mul_rn(dv, yi);   // y .= D_Dl1 .* y (:897) as the row is reached
                yk[li * S] = div_rn(sub_rn(yi, acc), dv);
            }
            if (!ok) break;
            if (wi > 0) {   // the pair's last, partly used chunk
                ++ch;
                rs.release(ch, lane);
            }
        }
        if (!ok) break;
        __syncwarp();
        {
            int pp = lane / ps, li = lane - pp * ps;
            for (int t = lane; t < nrows; t += 32) {
                y[rowbase + t] = (IO)ys[li * S + pp];
                li += dr;
                pp += dq;
                if (li >= ps) {
                    li -= ps;
                    ++pp;
                }
            }
        }
        __syncwarp();
    }
    if (!ok) {
        // A bounded wait ran out: record it, let the copies in flight land, and return.
        hsdev::cp_async_wait_all();
        if (lane == 0) hsdev::report_error(p.err, hsdev::kErrWaitTimeout);
        rs.drain();
    }
}

// Partsize PS known at compile time (8, 16): the row loop is unrolled, a
// lane's D_Dl1 stays in registers, x and y move as 16-byte vectors of the
// lane's own partition (rows contiguous), the row lists come in as broadcast
// words, and a lane only ever touches its own column of y in shared memory.
template <typename T, typename IO, int SWEEP, int PS>
__global__ void __launch_bounds__(kSegWarps * 32, 1) l1gs_seg_ps_kernel(const hsseg::Params p) {
    constexpr int S = 32;
    constexpr uint32_t SB = hsseg::slot_bytes(32, sizeof(T));
    constexpr int K = seg_k<T>();
    constexpr int NDIR = SWEEP == 2 ? 2 : 1;
    constexpr int PSQ = (PS + 3) & ~3;   // bytes of a group's row list
    constexpr int NW = PSQ / 4;
    constexpr int VX = 16 / (int)sizeof(IO), VD = 16 / (int)sizeof(T);
    static_assert(PS % VX == 0 && PS % VD == 0, "whole vectors per partition");
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wbase = smem + (size_t)warp * p.warp_bytes;
    T* yk = reinterpret_cast<T*>(wbase + p.ys_off) + lane;   // y of row li of the lane's partition: yk[li * S]; row PS: +0
    const T* __restrict__ D = static_cast<const T*>(p.D);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);
    const int wpb = blockDim.x >> 5;
    hsseg::SegStream<SB, K, NDIR, SWEEP> rs;
    rs.ring = wbase + p.ring_off;
    rs.bars = reinterpret_cast<uint64_t*>(wbase + p.bars_off);
    rs.tab = reinterpret_cast<TabEnt*>(wbase + p.tab_off);
    rs.nst = p.nst;
    rs.q0 = p.gbeg + blockIdx.x * wpb + warp;
    rs.qstride = gridDim.x * wpb;
    rs.lo = p.lo;
    rs.up = p.up;
    const int32_t my_groups = rs.q0 < p.gend ? (p.gend - 1 - rs.q0) / rs.qstride + 1 : 0;
    yk[PS * S] = T(0);
    rs.init(lane, my_groups);
    bool ok = true;
    int32_t ch = 0;   // chunk of the next slot
    for (int32_t gi = 0; gi < my_groups && ok; ++gi) {
        const int64_t g = rs.q0 + (int64_t)gi * rs.qstride;
        const int64_t prow = (g * 32 + lane) * (int64_t)PS;   // first row of the lane's partition
        const bool whole = p.vec_io && prow + PS <= p.n;
        T dreg[PS];
        if (whole) {
#pragma unroll
            for (int v = 0; v < PS / VX; ++v) {
                const uint4 w = *reinterpret_cast<const uint4*>(x + prow + v * VX);
                const IO* e = reinterpret_cast<const IO*>(&w);
#pragma unroll
                for (int c = 0; c < VX; ++c) yk[(v * VX + c) * S] = (T)e[c];
            }
#pragma unroll
            for (int v = 0; v < PS / VD; ++v) {
                const uint4 w = *reinterpret_cast<const uint4*>(D + prow + v * VD);
                const T* e = reinterpret_cast<const T*>(&w);
#pragma unroll
                for (int c = 0; c < VD; ++c) dreg[v * VD + c] = e[c];
            }
        } else {   // the short last partition, padding partitions, or unaligned vectors
#pragma unroll
            for (int li = 0; li < PS; ++li) {
                const bool valid = prow + li < p.n;
                yk[li * S] = valid ? (T)x[prow + li] : T(0);
                dreg[li] = valid ? D[prow + li] : T(1);
            }
        }
        // slots per row of each direction (the same words for every lane)
        uint32_t mw[NDIR][NW];
#pragma unroll
        for (int d = 0; d < NDIR; ++d)
#pragma unroll
            for (int w = 0; w < NW; ++w) mw[d][w] = reinterpret_cast<const uint32_t*>(rs.dir(d).maxc + g * PSQ)[w];
#pragma unroll
        for (int d = 0; d < NDIR; ++d) {
            const bool lowerdir = SWEEP == 0 || (SWEEP == 2 && d == 0);
            int wi = 0;   // slot of the next entry inside chunk ch
#pragma unroll
            for (int t = 0; t < PS; ++t) {
                const int li = lowerdir ? t : PS - 1 - t;
                const int m = (int)((mw[d][li >> 2] >> ((li & 3) * 8)) & 0xffu);
                T acc = T(0);
                for (int k = 0; k < m; ++k) {
                    if (ch >= rs.ready && !rs.wait_upto(ch)) {
                        ok = false;
                        break;
                    }
                    const unsigned char* sp = rs.slot(ch, wi);
                    const T a = reinterpret_cast<const T*>(sp)[lane];
                    const int col = reinterpret_cast<const uint16_t*>(sp + 32 * sizeof(T))[lane];
                    acc = add_rn(acc, mul_rn(a, yk[col * S]));
                    if (++wi == K) {   // a finished chunk goes back at once
                        wi = 0;
                        ++ch;
                        rs.release(ch, lane);
                    }
                }
                if (!ok) break;
                T yi = yk[li * S];
                if (SWEEP == 2 && !lowerdir) yi = mul_rn(dreg[li], yi);   // y .= D_Dl1 .* y (:897)
                yk[li * S] = div_rn(sub_rn(yi, acc), dreg[li]);
            }
            if (!ok) break;
            if (wi > 0) {   // the pair's last, partly used chunk
                ++ch;
                rs.release(ch, lane);
            }
        }
        if (!ok) break;
        if (whole) {
#pragma unroll
            for (int v = 0; v < PS / VX; ++v) {
                uint4 w;
                IO* e = reinterpret_cast<IO*>(&w);
#pragma unroll
                for (int c = 0; c < VX; ++c) e[c] = (IO)yk[(v * VX + c) * S];
                *reinterpret_cast<uint4*>(y + prow + v * VX) = w;
            }
        } else {
#pragma unroll
            for (int li = 0; li < PS; ++li)
                if (prow + li < p.n) y[prow + li] = (IO)yk[li * S];
        }
    }
    if (!ok) {
        if (lane == 0) hsdev::report_error(p.err, hsdev::kErrWaitTimeout);
        rs.drain();
    }
}

// Shared-memory slice of a warp: ring, barriers, table, y (+ D_Dl1 and the
// staged row counts for the runtime-partsize kernel).
template <typename T>
void seg_geometry(hsseg::Params& p, int G, bool with_d) {
    const uint32_t CHB = (uint32_t)(seg_k<T>() * (32 / G) * hsseg::slot_bytes(G, sizeof(T)));
    const uint32_t S = with_d ? G + 1 : 32;
    p.nst = 4;
    p.ring_off = 0;
    p.bars_off = p.nst * CHB;
    p.tab_off = (p.bars_off + 8 * p.nst + 15) / 16 * 16;
    p.ys_off = p.tab_off + kTab * (uint32_t)sizeof(TabEnt);
    p.ds_off = (p.ys_off + (uint32_t)(S * (p.ps + 1) * sizeof(T)) + 15) / 16 * 16;
    p.mx_off = (p.ds_off + (with_d ? (uint32_t)(S * p.ps * sizeof(T)) : 0u) + 15) / 16 * 16;
    const uint32_t psq = (uint32_t)((p.ps + 3) & ~3);
    p.warp_bytes = (p.mx_off + (with_d ? 2 * psq : 0u) + 127) / 128 * 128;
}

template <typename K>
int launch_kernel(K kern, hsseg::Params& p, cudaStream_t st) {
    int best_w = 0, best_warps = 0, best_per_sm = 0;
    for (int w = kSegWarps; w >= 1; w >>= 1) {
        const size_t smem = (size_t)w * p.warp_bytes;
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
    const int64_t ngr = (int64_t)p.gend - p.gbeg;
    const int64_t slots = (int64_t)best_per_sm * hs::num_sms() * best_w;
    const int64_t rounds = std::max<int64_t>(1, (ngr + slots - 1) / slots);
    const int64_t grid = std::max<int64_t>(1, (ngr + rounds * best_w - 1) / (rounds * best_w));
    kern<<<(int)grid, best_w * 32, (size_t)best_w * p.warp_bytes, st>>>(p);
    HS_LAUNCH_CHECK("l1gs_seg_kernel");
    return HS_OK;
}

template <typename T, typename IO, int SWEEP>
int launch_t(const hsseg::View& view, hsseg::Params& p, cudaStream_t st) {
    (void)view;
    switch (p.ps) {
        case 8:
            if (p.G == 32) {
                seg_geometry<T>(p, 32, false);
                return launch_kernel(l1gs_seg_ps_kernel<T, IO, SWEEP, 8>, p, st);
            }
            break;
        case 16:
            if (p.G == 32) {
                seg_geometry<T>(p, 32, false);
                return launch_kernel(l1gs_seg_ps_kernel<T, IO, SWEEP, 16>, p, st);
            }
            break;
        default: break;
    }
    seg_geometry<T>(p, p.G, true);
    switch (p.G) {
        case 32: return launch_kernel(l1gs_seg_kernel<T, IO, SWEEP, 32>, p, st);
        case 16: return launch_kernel(l1gs_seg_kernel<T, IO, SWEEP, 16>, p, st);
        case 8: return launch_kernel(l1gs_seg_kernel<T, IO, SWEEP, 8>, p, st);
        default: return launch_kernel(l1gs_seg_kernel<T, IO, SWEEP, 4>, p, st);
    }
}

template <typename T, typename IO>
int launch_io(int sweep, const hsseg::View& view, hsseg::Params& p, cudaStream_t st) {
    switch (sweep) {
        case HS_SWEEP_FORWARD: return launch_t<T, IO, 0>(view, p, st);
        case HS_SWEEP_BACKWARD: return launch_t<T, IO, 1>(view, p, st);
        default: return launch_t<T, IO, 2>(view, p, st);
    }
}

}  // namespace

namespace hsseg {

template <typename TM, typename TS>
int build(int32_t n, int32_t ps, int32_t nparts, const int32_t* rp, const int32_t* ci, const TM* v, bool lower,
          bool upper, View* view, cudaStream_t st) {
    if (ps > kMaxPartsize) return hs::set_error(HS_ERR_UNSUPPORTED, "segment lists need partsize <= %d", kMaxPartsize);
    const int32_t G = pick_group(ps, sizeof(TS));
    const int32_t ngroups = (int32_t)(((int64_t)nparts + G - 1) / G);
    const int32_t psq = (ps + 3) & ~3;
    view->G = G;
    view->ngroups = ngroups;
    const int64_t items = (int64_t)ngroups * ps;
    Tmp tmp;
    int32_t *cntL = nullptr, *qL = nullptr, *cntU = nullptr, *qU = nullptr;
    uint16_t* off = nullptr;
    int rc;
    if ((rc = tmp.get(&cntL, 4 * (size_t)n)) || (rc = tmp.get(&qL, 4 * (size_t)n)) ||
        (rc = tmp.get(&cntU, 4 * (size_t)n)) || (rc = tmp.get(&qU, 4 * (size_t)n)) ||
        (rc = tmp.get(&off, 2 * (size_t)items)))
        return rc;
    seg_count_kernel<<<grid_of(n), 256, 0, st>>>(n, ps, rp, ci, cntL, qL, cntU, qU);
    HS_LAUNCH_CHECK("seg_count_kernel");
    const int64_t SB = hsseg::slot_bytes(G, sizeof(TS));
    for (int d = 0; d < 2; ++d) {
        if ((d == 0 && !lower) || (d == 1 && !upper)) continue;
        Dir& dd = d == 0 ? view->lo : view->up;
        const int32_t* cnt = d == 0 ? cntL : cntU;
        const int32_t* q0 = d == 0 ? qL : qU;
        if ((rc = dalloc(view, &dd.maxc, (size_t)ngroups * psq)) || (rc = dalloc(view, &dd.total, 4 * (size_t)ngroups)) ||
            (rc = dalloc(view, &dd.base, 8 * (size_t)ngroups)))
            return rc;
        HS_CUDA(cudaMemsetAsync(dd.maxc, 0, (size_t)ngroups * psq, st));
        seg_max_kernel<<<grid_of(items * 32), 256, 0, st>>>(n, ps, psq, G, nparts, items, cnt, dd.maxc);
        HS_LAUNCH_CHECK("seg_max_kernel");
        seg_off_kernel<<<grid_of(ngroups), 256, 0, st>>>(ngroups, ps, psq, dd.maxc, off, dd.total, d == 1);
        HS_LAUNCH_CHECK("seg_off_kernel");
        std::vector<int32_t> tot(ngroups);
        std::vector<int64_t> base(ngroups);
        HS_CUDA(cudaMemcpyAsync(tot.data(), dd.total, 4 * (size_t)ngroups, cudaMemcpyDeviceToHost, st));
        HS_CUDA(cudaStreamSynchronize(st));
        int64_t acc = 0;
        for (int32_t g = 0; g < ngroups; ++g) {
            base[g] = acc;
            acc += tot[g];
        }
        dd.slots = acc;
        HS_CUDA(cudaMemcpyAsync(dd.base, base.data(), 8 * (size_t)ngroups, cudaMemcpyHostToDevice, st));
        if ((rc = dalloc(view, &dd.stream, (size_t)(acc * SB)))) return rc;
        HS_CUDA(cudaMemsetAsync(dd.stream, 0, (size_t)(acc * SB), st));
        if (acc > 0) {
            seg_pad_kernel<TS><<<grid_of(acc * G), 256, 0, st>>>(acc, ps, G, dd.stream);
            HS_LAUNCH_CHECK("seg_pad_kernel");
        }
        seg_scatter_kernel<TM, TS><<<grid_of(n), 256, 0, st>>>(n, ps, G, ci, v, cnt, q0, off, dd.base, dd.stream);
        HS_LAUNCH_CHECK("seg_scatter_kernel");
        HS_CUDA(cudaStreamSynchronize(st));   // the host base vector and the scratch go out of scope
    }
    return HS_OK;
}

template int build<double, double>(int32_t, int32_t, int32_t, const int32_t*, const int32_t*, const double*, bool,
                                   bool, View*, cudaStream_t);
template int build<double, float>(int32_t, int32_t, int32_t, const int32_t*, const int32_t*, const double*, bool,
                                  bool, View*, cudaStream_t);
template int build<float, float>(int32_t, int32_t, int32_t, const int32_t*, const int32_t*, const float*, bool, bool,
                                 View*, cudaStream_t);

void destroy(View* view) {
    for (Dir* dd : {&view->lo, &view->up}) {
        cudaFree(dd->stream);
        cudaFree(dd->base);
        cudaFree(dd->total);
        cudaFree(dd->maxc);
        *dd = Dir();
    }
    view->bytes = 0;
}

int launch(int sdt, int io, int sweep, const View& view, int32_t n, int32_t ps, int32_t gbeg, int32_t gend,
           const void* D, const void* x, void* y, int32_t* err, cudaStream_t st) {
    if (gend <= gbeg) return HS_OK;
    Params p;
    p.n = n;
    p.ps = ps;
    p.gbeg = gbeg;
    p.gend = gend;
    p.lo = view.lo;
    p.up = view.up;
    p.D = D;
    p.x = x;
    p.y = y;
    p.err = err;
    p.G = view.G;
    p.vec_io = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y) | reinterpret_cast<uintptr_t>(D)) & 15u) == 0;
    if (sdt == HS_F64 && io == HS_F64) return launch_io<double, double>(sweep, view, p, st);
    if (sdt == HS_F32 && io == HS_F32) return launch_io<float, float>(sweep, view, p, st);
    if (sdt == HS_F32 && io == HS_F64) return launch_io<float, double>(sweep, view, p, st);
    return hs::set_error(HS_ERR_UNSUPPORTED, "FP64 smoother with FP32 vectors is not provided");
}

}  // namespace hsseg
