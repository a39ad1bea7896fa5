// Matrix-view L1 Gauss-Seidel over per-group segment lists: build and apply
// (layout and order of operations: l1gs_seg.cuh).
#include <algorithm>
#include <vector>

#include "l1gs_seg.cuh"

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

// One warp per (group, row): the lanes' counts (interleaved) and their maximum.
__global__ void seg_max_kernel(int32_t n, int32_t ps, int32_t nparts, int64_t items, const int32_t* __restrict__ cnt,
                               uint8_t* __restrict__ maxc, uint8_t* __restrict__ cnti) {
    const int lane = threadIdx.x & 31;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < items;
         w += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t g = w / ps, li = w - g * ps;
        const int64_t k = g * 32 + lane, row = k * ps + li;
        const int32_t c = (k < nparts && row < n) ? cnt[row] : 0;
        const unsigned m = __reduce_max_sync(FULL, (unsigned)c);
        cnti[w * 32 + lane] = (uint8_t)c;
        if (lane == 0) maxc[w] = (uint8_t)m;
    }
}

// Per group: the first slot of every row in the sweep's row order (ascending
// rows for the lower lists, descending for the upper), and the group's total.
__global__ void seg_off_kernel(int32_t ngroups, int32_t ps, const uint8_t* __restrict__ maxc,
                               uint16_t* __restrict__ off, int32_t* __restrict__ total, int descending) {
    for (int32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x) {
        int32_t acc = 0;
        for (int32_t t = 0; t < ps; ++t) {
            const int64_t li = descending ? ps - 1 - t : t;
            off[(int64_t)g * ps + li] = (uint16_t)acc;
            acc += maxc[(int64_t)g * ps + li];
        }
        total[g] = acc;
    }
}

template <typename TM, typename TS>
__global__ void seg_scatter_kernel(int32_t n, int32_t ps, const int32_t* __restrict__ ci, const TM* __restrict__ v,
                                   const int32_t* __restrict__ cnt, const int32_t* __restrict__ q0,
                                   const uint16_t* __restrict__ off, const int64_t* __restrict__ base,
                                   unsigned char* __restrict__ stream) {
    constexpr int64_t SB = 32 * (sizeof(TS) + 2);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / ps, li = i - k * ps, g = k / 32, lane = k - g * 32, s = k * ps;
        const int64_t slot0 = base[g] + off[g * ps + li];
        for (int32_t t = 0; t < cnt[i]; ++t) {
            const int32_t q = q0[i] + t;
            unsigned char* sp = stream + (slot0 + t) * SB;
            reinterpret_cast<TS*>(sp)[lane] = (TS)v[q];
            reinterpret_cast<uint16_t*>(sp + 32 * sizeof(TS))[lane] = (uint16_t)(ci[q] - s);
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
template <typename T, typename IO, int SWEEP>
__global__ void __launch_bounds__(kSegWarps * 32) l1gs_seg_kernel(const hsseg::Params p) {
    constexpr int S = 33;
    constexpr uint32_t SB = 32 * (sizeof(T) + 2);                 // bytes per slot
    constexpr uint32_t K = hsseg::kSlotsPerChunk(sizeof(T));      // slots per chunk
    constexpr uint32_t CHB = K * SB;                              // bytes per chunk
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ps = p.ps;
    const uint32_t nst = p.nst;
    unsigned char* wbase = smem + (size_t)warp * p.warp_bytes;
    unsigned char* ring = wbase + p.ring_off;
    uint64_t* bars = reinterpret_cast<uint64_t*>(wbase + p.bars_off);
    T* ys = reinterpret_cast<T*>(wbase + p.ys_off);   // y of row li, lane's partition: ys[li * S + lane]
    T* ds = reinterpret_cast<T*>(wbase + p.ds_off);
    const T* __restrict__ D = static_cast<const T*>(p.D);
    const IO* __restrict__ x = static_cast<const IO*>(p.x);
    IO* __restrict__ y = static_cast<IO*>(p.y);
    const int wpb = blockDim.x >> 5;
    const int32_t q0 = p.gbeg + blockIdx.x * wpb + warp, qstride = gridDim.x * wpb;
    const int32_t my_groups = q0 < p.gend ? (p.gend - 1 - q0) / qstride + 1 : 0;
    constexpr int NDIR = SWEEP == 2 ? 2 : 1;
    auto dir_of = [&](int d) -> const hsseg::Dir& { return (SWEEP == 1 || d == 1) ? p.up : p.lo; };

    // Producer (lane 0): walks (group, direction, chunk) of this warp's streams.
    int32_t issued = 0, pgi = 0, pd = 0, pc = 0, pnch = -1;
    const unsigned char* psrc = nullptr;
    int32_t ptot = 0;
    auto advance = [&]() -> bool {   // position on the next non-empty (group, direction); false at the end
        while (pgi < my_groups) {
            if (pnch < 0) {
                const int64_t g = q0 + (int64_t)pgi * qstride;
                const hsseg::Dir& dd = dir_of(pd);
                ptot = dd.total[g];
                pnch = (int32_t)((ptot + K - 1) / K);
                psrc = dd.stream + dd.base[g] * SB;
                pc = 0;
            }
            if (pc < pnch) return true;
            pnch = -1;
            if (++pd == NDIR) {
                pd = 0;
                ++pgi;
            }
        }
        return false;
    };
    auto issue_next = [&]() -> bool {
        if (!advance()) return false;
        const uint32_t s = (uint32_t)issued & (nst - 1u);
        const uint32_t bytes = (uint32_t)min((int32_t)K, ptot - pc * (int32_t)K) * SB;
        hsdev::mbar_arrive_expect_tx(bars + s, bytes);
        hsdev::bulk_load(ring + (size_t)s * CHB, psrc + (size_t)pc * CHB, bytes, bars + s);
        ++issued;
        ++pc;
        return true;
    };
    int32_t total = 0;   // chunks of all this warp's streams (each lane counts)
    for (int32_t gi = 0; gi < my_groups; ++gi)
        for (int d = 0; d < NDIR; ++d) total += (dir_of(d).total[q0 + (int64_t)gi * qstride] + K - 1) / K;
    if (lane == 0) {
        for (uint32_t s = 0; s < nst; ++s) hsdev::mbar_init(bars + s, 1);
        hsdev::fence_barrier_init();
        while (issued < total && issued < (int32_t)nst) issue_next();
    }
    __syncwarp();
    int32_t ready = 0, freed = 0;
    bool ok = true;
    auto wait_upto = [&](int32_t last) -> bool {
        while (ready <= last) {
            const bool got = hsdev::mbar_wait_bounded(bars + ((uint32_t)ready & (nst - 1u)), ((uint32_t)ready / nst) & 1u);
            if (!__all_sync(FULL, got)) return false;
            ++ready;
        }
        return true;
    };
    auto release = [&](int32_t upto) {
        if (upto <= freed) return;
        freed = upto;
        __syncwarp();
        if (lane == 0) {
            hsdev::fence_proxy_async_smem();
            while (issued < total && issued < freed + (int32_t)nst) issue_next();
        }
    };

    int32_t cbase = 0;   // first chunk of the current (group, direction)
    for (int32_t gi = 0; gi < my_groups && ok; ++gi) {
        const int64_t g = q0 + (int64_t)gi * qstride;
        const int64_t rowbase = g * 32 * (int64_t)ps;
        {   // x and D_Dl1 of the group's rows -> [li][partition], coalesced
            int pp = lane / ps, li = lane - (lane / ps) * ps;
            for (int t = lane; t < 32 * ps; t += 32) {
                const int64_t row = rowbase + t;
                const bool valid = row < p.n;
                ys[li * S + pp] = valid ? (T)x[row] : T(0);
                ds[li * S + pp] = valid ? D[row] : T(1);
                li += 32;
                while (li >= ps) {
                    li -= ps;
                    ++pp;
                }
            }
        }
        __syncwarp();
        T* yk = ys + lane;
        const T* dk = ds + lane;
        for (int d = 0; d < NDIR && ok; ++d) {
            const bool lowerdir = SWEEP == 0 || (SWEEP == 2 && d == 0);
            const hsseg::Dir& dd = lowerdir ? p.lo : p.up;
            const int32_t nch = (dd.total[g] + (int32_t)K - 1) / (int32_t)K;
            const uint8_t* __restrict__ mx = dd.maxc + g * ps;
            const uint16_t* __restrict__ of = dd.off + g * ps;
            const uint8_t* __restrict__ cn = dd.cnt + g * ps * 32 + lane;
            for (int t = 0; t < ps; ++t) {
                const int li = lowerdir ? t : ps - 1 - t;
                const int m = __ldg(mx + li);
                const int o = __ldg(of + li);
                const int c = __ldg(cn + li * 32);
                T acc = T(0);
                for (int k = 0; k < m; ++k) {
                    const int32_t slot = o + k;
                    const int32_t chunk = cbase + slot / (int32_t)K;
                    if (chunk >= ready && !wait_upto(chunk)) {
                        ok = false;
                        break;
                    }
                    if (k < c) {
                        const unsigned char* sp =
                            ring + (size_t)((uint32_t)chunk & (nst - 1u)) * CHB + (size_t)(slot % (int32_t)K) * SB;
                        const T a = reinterpret_cast<const T*>(sp)[lane];
                        const int col = reinterpret_cast<const uint16_t*>(sp + 32 * sizeof(T))[lane];
                        acc = add_rn(acc, mul_rn(a, yk[col * S]));
                    }
                    // a finished chunk goes back at once: a row may span more chunks than the ring holds
                    if ((slot + 1) % (int32_t)K == 0) release(cbase + (slot + 1) / (int32_t)K);
                }
                if (!ok) break;
                const T dv = dk[li * S];
                T yi = yk[li * S];
                if (SWEEP == 2 && !lowerdir) yi = mul_rn(dv, yi);   // y .= D_Dl1 .* y (:897) as the row is reached
                yk[li * S] = div_rn(sub_rn(yi, acc), dv);
            }
            if (!ok) break;
            release(cbase + nch);
            cbase += nch;
        }
        if (!ok) break;
        __syncwarp();
        {
            int pp = lane / ps, li = lane - (lane / ps) * ps;
            for (int t = lane; t < 32 * ps; t += 32) {
                const int64_t row = rowbase + t;
                if (row < p.n) y[row] = (IO)ys[li * S + pp];
                li += 32;
                while (li >= ps) {
                    li -= ps;
                    ++pp;
                }
            }
        }
        __syncwarp();
    }
    if (!ok) {
        if (lane == 0) hsdev::report_error(p.err, hsdev::kErrWaitTimeout);
        const int32_t end = __shfl_sync(FULL, issued, 0);
        for (int32_t c = ready; c < end; ++c)
            (void)hsdev::mbar_wait_bounded(bars + ((uint32_t)c & (nst - 1u)), ((uint32_t)c / nst) & 1u);
    }
}

template <typename T, typename IO, int SWEEP>
int launch_t(const hsseg::View& view, hsseg::Params& p, cudaStream_t st) {
    constexpr uint32_t CHB = hsseg::kSlotsPerChunk(sizeof(T)) * 32 * (sizeof(T) + 2);
    p.nst = 4;
    p.ring_off = 0;
    p.bars_off = p.nst * CHB;
    p.ys_off = (p.bars_off + 8 * p.nst + 15) / 16 * 16;
    const uint32_t slice = (uint32_t)(33 * p.ps * sizeof(T));
    p.ds_off = (p.ys_off + slice + 15) / 16 * 16;
    p.warp_bytes = (p.ds_off + slice + 127) / 128 * 128;
    auto kern = l1gs_seg_kernel<T, IO, SWEEP>;
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
    (void)view;
    return HS_OK;
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
    const int32_t ngroups = (int32_t)(((int64_t)nparts + 31) / 32);
    view->ngroups = ngroups;
    const int64_t items = (int64_t)ngroups * ps;
    Tmp tmp;
    int32_t *cntL = nullptr, *qL = nullptr, *cntU = nullptr, *qU = nullptr;
    int rc;
    if ((rc = tmp.get(&cntL, 4 * (size_t)n)) || (rc = tmp.get(&qL, 4 * (size_t)n)) ||
        (rc = tmp.get(&cntU, 4 * (size_t)n)) || (rc = tmp.get(&qU, 4 * (size_t)n)))
        return rc;
    seg_count_kernel<<<grid_of(n), 256, 0, st>>>(n, ps, rp, ci, cntL, qL, cntU, qU);
    HS_LAUNCH_CHECK("seg_count_kernel");
    constexpr int64_t SB = 32 * (sizeof(TS) + 2);
    for (int d = 0; d < 2; ++d) {
        if ((d == 0 && !lower) || (d == 1 && !upper)) continue;
        Dir& dd = d == 0 ? view->lo : view->up;
        const int32_t* cnt = d == 0 ? cntL : cntU;
        const int32_t* q0 = d == 0 ? qL : qU;
        if ((rc = dalloc(view, &dd.maxc, (size_t)items)) || (rc = dalloc(view, &dd.cnt, 32 * (size_t)items)) ||
            (rc = dalloc(view, &dd.off, 2 * (size_t)items)) || (rc = dalloc(view, &dd.total, 4 * (size_t)ngroups)) ||
            (rc = dalloc(view, &dd.base, 8 * (size_t)ngroups)))
            return rc;
        seg_max_kernel<<<grid_of(items * 32), 256, 0, st>>>(n, ps, nparts, items, cnt, dd.maxc, dd.cnt);
        seg_off_kernel<<<grid_of(ngroups), 256, 0, st>>>(ngroups, ps, dd.maxc, dd.off, dd.total, d == 1);
        hs::count_launch();
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
        seg_scatter_kernel<TM, TS><<<grid_of(n), 256, 0, st>>>(n, ps, ci, v, cnt, q0, dd.off, dd.base, dd.stream);
        HS_LAUNCH_CHECK("seg_scatter_kernel");
        HS_CUDA(cudaStreamSynchronize(st));   // the host base vector goes out of scope
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
        cudaFree(dd->off);
        cudaFree(dd->maxc);
        cudaFree(dd->cnt);
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
    if (sdt == HS_F64 && io == HS_F64) return launch_io<double, double>(sweep, view, p, st);
    if (sdt == HS_F32 && io == HS_F32) return launch_io<float, float>(sweep, view, p, st);
    if (sdt == HS_F32 && io == HS_F64) return launch_io<float, double>(sweep, view, p, st);
    return hs::set_error(HS_ERR_UNSUPPORTED, "FP64 smoother with FP32 vectors is not provided");
}

}  // namespace hsseg
