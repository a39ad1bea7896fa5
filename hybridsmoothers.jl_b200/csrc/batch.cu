// Batched, served PCG for many independent systems on one B200.
//
// Every admitted system ("slot") keeps its FP64 CSR matrix, its FP32 L1GS
// symmetric packed preconditioner and its Krylov state (x, r, z, p, q and the
// scalars) resident in HBM until it converges.  One batched PCG iteration
// advances all active slots with a fixed number of launches, independent of
// how many slots are active:
//   seg_spmv_dot  q = A p and per-block partials of p.q      (all slots)
//   seg_alpha     alpha = rz / pq                            (one block per slot)
//   seg_update    x += alpha p, r -= alpha q, partials of r.r
//   seg_check     convergence test, iteration count
//   l1gs_batched  z = M^-1 r and per-item partials of r.z, one launch per partsize class
//                 (FP32 smoother, FP64 in/out)
//   seg_beta      beta = rz_new / rz (r.z partials come from the L1GS apply)
//   seg_p         p = z + beta p
// The iteration is captured once as a CUDA graph per active set and replayed.
// A slot's reductions always use the same blocks over its own rows and a
// fixed-order finalize, so a slot's iterates are bitwise the same whether it
// runs alone or among others.
//
// Admission (hs_batch_submit) builds the slot on a setup stream; called
// between hs_batch_launch and hs_batch_wait it overlaps the running
// iterations, and the new system joins at the next launch.  A request is
// refused with HS_ERR_BUDGET until a slot and enough of the HBM budget are
// free.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "reduce.cuh"
#include "spmv.cuh"

namespace {

constexpr int kRPB = 256;     // rows per CSR-stream pass (= threads per CTA)
constexpr int kSub = 4;       // passes per CTA
constexpr int kRPC = kRPB * kSub;   // rows per CTA of the segmented kernels
constexpr int kT = 256;
constexpr int kBatchE = 16;   // stream rows per tile of the batched smoother

struct Scalars {
    double bb, rr, rz, pq, alpha, beta, rtol;
    int done, it, conv_it, active;
};

using hsdev::DD;

__device__ __forceinline__ void store_dd(double* partials, DD v) {
    v = hsdev::block_dd(v);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = v.s;
        partials[2 * blockIdx.x + 1] = v.c;
    }
}

// Per slot: its CTA range (for the per-slot reductions) and scalars.
struct SlotDev {
    int32_t n, blk0, nblk, item0, nitems, ps;
    Scalars* s;
};

// One CTA of the segmented vector kernels: kRPC rows of one slot, with every
// pointer it needs, so a CTA starts after one load of its entry.
struct BlockMap {
    int32_t n, row0;
    const int64_t* soff;   // the slot's matrix in 32-row slices (spmv.cuh): first entry of each
    const int32_t* scol;
    const double* sval;
    double *x, *r, *z, *p, *q;
    const Scalars* s;
};

// One work item of the batched L1GS apply: 32 partitions (a group) of a slot,
// with its stream bases, D_Dl1 and vectors already offset to the group.
struct PrecItem {
    const float* ST;   // the group's tile stream: lower tiles, then upper tiles (E x 32 floats each)
    const float* Di;
    const double* x;   // r of the group's first row
    double* y;         // z likewise
    int64_t npad;
    int32_t rows;      // rows of the slot from the group's first row on
    int32_t tlen;
    const Scalars* s;
};

// ---- segmented PCG kernels --------------------------------------------------
// Same arithmetic as the single-system driver: compensated (Dot2) dots,
// separately rounded updates, storage-order SpMV rows.  The streaming kernels
// load kSub elements per thread before using any.
__global__ void __launch_bounds__(kT, 4) seg_spmv_dot(const BlockMap* __restrict__ map, double* __restrict__ partials) {
    const BlockMap m = map[blockIdx.x];
    DD part{0.0, 0.0};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // The slice bounds of all the warp's slices, requested before the slot's
    // flag is known.
    constexpr int NS = kRPC / kT;
    int64_t o0[NS], o1[NS];
    const int64_t nsl = ((int64_t)m.n + 31) / 32;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const int64_t sl = ((int64_t)m.row0 >> 5) + k * (kT / 32) + warp;
        o0[k] = sl < nsl ? m.soff[sl] : 0;
        o1[k] = sl < nsl ? m.soff[sl + 1] : 0;
    }
    if (!m.s->done) {   // uniform over the CTA (one slot per CTA)
        auto fp = [&](int32_t j) { return __ldg(m.p + j); };
#pragma unroll
        for (int k = 0; k < NS; ++k) {   // the warp's 32-row slices of this CTA
            const int64_t row0 = (int64_t)m.row0 + (k * (kT / 32) + warp) * 32;
            if (row0 >= m.n) break;   // uniform over the warp
            const double acc = hsdev::slice_row_sum(o0[k], o1[k], m.scol, m.sval, fp);
            const int64_t r = row0 + lane;
            if (r < m.n) {
                m.q[r] = acc;
                hsdev::dd_add_prod(part, m.p[r], acc);
            }
        }
    }
    store_dd(partials, part);
}

// Sum of a slot's CTA partials (valid on thread 0).  A large slot has
// thousands of CTAs: each thread loads 8 partials before adding any.
__device__ __forceinline__ double range_sum(const double* __restrict__ partials, int32_t first, int32_t count) {
    DD v{0.0, 0.0};
    const double2* p2 = reinterpret_cast<const double2*>(partials) + first;
    for (int base = threadIdx.x; base < count; base += 8 * blockDim.x) {
        double2 w[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (base + k * (int)blockDim.x < count) w[k] = p2[base + k * blockDim.x];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (base + k * (int)blockDim.x < count) v = hsdev::dd_add(v, DD{w[k].x, w[k].y});
    }
    return hsdev::dd_value(hsdev::block_dd(v));
}
__device__ __forceinline__ double slot_sum(const double* __restrict__ partials, const SlotDev& sd) {
    return range_sum(partials, sd.blk0, sd.nblk);
}

__global__ void seg_alpha(const SlotDev* __restrict__ slots, const int32_t* __restrict__ active,
                          const double* __restrict__ partials) {
    const SlotDev sd = slots[active[blockIdx.x]];
    const double pq = slot_sum(partials, sd);
    if (threadIdx.x == 0 && !sd.s->done) {
        sd.s->pq = pq;
        sd.s->alpha = __ddiv_rn(sd.s->rz, pq);
    }
}

__global__ void __launch_bounds__(kT) seg_update(const BlockMap* __restrict__ map, double* __restrict__ partials) {
    const BlockMap m = map[blockIdx.x];
    DD part{0.0, 0.0};
    if (!m.s->done) {
        const double alpha = m.s->alpha;
        double xv[kSub], pv[kSub], rv[kSub], qv[kSub];
#pragma unroll
        for (int k = 0; k < kSub; ++k) {
            const int i = m.row0 + k * kRPB + threadIdx.x;
            if (i < m.n) {
                xv[k] = m.x[i];
                pv[k] = m.p[i];
                rv[k] = m.r[i];
                qv[k] = m.q[i];
            }
        }
#pragma unroll
        for (int k = 0; k < kSub; ++k) {
            const int i = m.row0 + k * kRPB + threadIdx.x;
            if (i < m.n) {
                m.x[i] = __dadd_rn(xv[k], __dmul_rn(alpha, pv[k]));
                const double ri = __dsub_rn(rv[k], __dmul_rn(alpha, qv[k]));
                m.r[i] = ri;
                hsdev::dd_add_prod(part, ri, ri);
            }
        }
    }
    store_dd(partials, part);
}

__global__ void seg_check(const SlotDev* __restrict__ slots, const int32_t* __restrict__ active,
                          const double* __restrict__ partials, int32_t maxit) {
    const SlotDev sd = slots[active[blockIdx.x]];
    const double rr = slot_sum(partials, sd);
    if (threadIdx.x == 0 && !sd.s->done) {
        Scalars* s = sd.s;
        s->it += 1;
        s->rr = rr;
        if (sqrt(rr) <= __dmul_rn(s->rtol, sqrt(s->bb))) {
            s->done = 1;
            s->conv_it = s->it;
        } else if (s->it >= maxit) {
            s->done = 2;   // gave up
            s->conv_it = s->it;
        }
    }
}

// r.z of the slot: the batched L1GS apply leaves one compensated partial per
// work item (the slot's items are contiguous).
__global__ void seg_beta(const SlotDev* __restrict__ slots, const int32_t* __restrict__ active,
                         const double* __restrict__ rz_part) {
    const SlotDev sd = slots[active[blockIdx.x]];
    const double rz = range_sum(rz_part, sd.item0, sd.nitems);
    if (threadIdx.x == 0 && !sd.s->done) {
        sd.s->beta = __ddiv_rn(rz, sd.s->rz);
        sd.s->rz = rz;
    }
}

__global__ void __launch_bounds__(kT) seg_p(const BlockMap* __restrict__ map) {
    const BlockMap m = map[blockIdx.x];
    if (m.s->done) return;
    const double beta = m.s->beta;
    double zv[kSub], pv[kSub];
#pragma unroll
    for (int k = 0; k < kSub; ++k) {
        const int i = m.row0 + k * kRPB + threadIdx.x;
        if (i < m.n) {
            zv[k] = m.z[i];
            pv[k] = m.p[i];
        }
    }
#pragma unroll
    for (int k = 0; k < kSub; ++k) {
        const int i = m.row0 + k * kRPB + threadIdx.x;
        if (i < m.n) m.p[i] = __dadd_rn(zv[k], __dmul_rn(beta, pv[k]));
    }
}

// Slot initialisation after admission: x = 0, r = b, bb = b.b (z, p, rz after the first apply)
__global__ void init_vectors(int32_t n, const double* __restrict__ b, double* __restrict__ x, double* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = 0.0;
        r[i] = b[i];
    }
}

__global__ void init_p_partials(int32_t n, const double* __restrict__ z, double* __restrict__ p,
                                const double* __restrict__ r, const double* __restrict__ b,
                                double* __restrict__ pbb, double* __restrict__ prz) {
    DD bb{0.0, 0.0}, rz{0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        p[i] = z[i];
        hsdev::dd_add_prod(bb, b[i], b[i]);
        hsdev::dd_add_prod(rz, r[i], z[i]);
    }
    store_dd(pbb, bb);
    __syncthreads();
    store_dd(prz, rz);
}

__global__ void init_scalars(const double* __restrict__ pbb, const double* __restrict__ prz, int nb, Scalars* s,
                             double rtol) {
    DD vb{0.0, 0.0}, vr{0.0, 0.0};
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        vb = hsdev::dd_add(vb, DD{pbb[2 * i], pbb[2 * i + 1]});
        vr = hsdev::dd_add(vr, DD{prz[2 * i], prz[2 * i + 1]});
    }
    const double bb = hsdev::dd_value(hsdev::block_dd(vb));
    __syncthreads();
    const double rz = hsdev::dd_value(hsdev::block_dd(vr));
    if (threadIdx.x == 0) {
        s->bb = bb;
        s->rr = bb;
        s->rz = rz;
        s->rtol = rtol;
        s->done = bb == 0.0 ? 1 : 0;
        s->it = 0;
        s->conv_it = s->done ? 0 : -1;
        s->active = 1;
    }
}

// ---- batched L1GS symmetric apply (FP32 smoother, FP64 vectors) -----------
// Work item -> 32 partitions (a group) of one slot, one lane each.  At
// admission the slot's packed triangles are regrouped so that each group's
// tiles (E stream rows x 32 partitions, lower then upper, the last tile of
// each triangle padded with zeros) are contiguous: a tile is one 1D bulk copy
// of E x 128 bytes into the per-warp ring.  y and D_Dl1 live in registers,
// exactly like the single-system partsize<=32 kernel; the sums read only the
// triangle's entries, so the padding is never added.  The elected lane keeps
// the tile stream of the item it is issuing for in a register.  Tiles of
// converged slots are still fetched and applied until they leave the tables
// at the next rebuild.
template <int E>
__global__ void batch_tiles_kernel(int64_t ngroups, int32_t tlen, int32_t nt, int64_t npad,
                                   const float* __restrict__ SLi, const float* __restrict__ SUi,
                                   float* __restrict__ tiles) {
    const int64_t per_group = (int64_t)2 * nt * E * 32;
    const int64_t total = ngroups * per_group;
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < total;
         o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = o / per_group;
        const int64_t w = o - g * per_group;
        const int64_t t = w / (E * 32), rem = w - t * (E * 32);
        const int64_t row = rem / 32, lane = rem - row * 32;
        const bool upper = t >= nt;
        const int64_t e = (upper ? t - nt : t) * E + row;
        tiles[o] = e < tlen ? (upper ? SUi : SLi)[e * npad + g * 32 + lane] : 0.0f;
    }
}

template <int PS, int E, int STAGES>
__global__ void __launch_bounds__(128, 3)
    l1gs_batched_kernel(const PrecItem* __restrict__ items, int32_t nitems, double* __restrict__ rz_part,
                        int32_t* err) {
    constexpr int TLEN = PS * (PS - 1) / 2;
    constexpr int NT = (TLEN + E - 1) / E;
    constexpr int NTPG = 2 * NT;
    constexpr int XS = PS + 1;
    static_assert(PS % 2 == 0, "even partsize");
    static_assert(E <= 32, "one lane per tile row");
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr uint32_t kRing = E * 32 * 4 * STAGES;
    constexpr uint32_t kWarpBytes = (kRing + 8 * STAGES + 32 * XS * 4 + 127) / 128 * 128;
    unsigned char* wbase = smem + (size_t)warp * kWarpBytes;
    float* ring = reinterpret_cast<float*>(wbase);
    uint64_t* bars = reinterpret_cast<uint64_t*>(wbase + kRing);
    float* xs = reinterpret_cast<float*>(wbase + kRing + 8 * STAGES);
    const int wpb = blockDim.x >> 5;
    const int32_t w0 = blockIdx.x * wpb + warp, wstride = gridDim.x * wpb;
    const int32_t my_items = w0 < nitems ? (nitems - 1 - w0) / wstride + 1 : 0;
    const int32_t total = my_items * NTPG;

    // Tile refills: lane 0 copies the tile (E x 128 contiguous bytes) with one
    // bulk copy onto the stage's barrier.  It keeps the tile stream of the
    // item it issues for (one load per item).
    int32_t cache_ii = -1;
    const float* cST = nullptr;
    auto issue = [&](int32_t c) {   // called by lane 0
        const int32_t ii = c / NTPG;
        if (ii != cache_ii) {
            cST = items[w0 + ii * wstride].ST;
            cache_ii = ii;
        }
        const int32_t ti = c - ii * NTPG;
        const int stage = c & (STAGES - 1);
        uint64_t* bar = bars + stage;
        hsdev::mbar_arrive_expect_tx(bar, (uint32_t)(E * 32 * 4));
        hsdev::bulk_load(ring + stage * (E * 32), cST + (int64_t)ti * E * 32, (uint32_t)(E * 32 * 4), bar);
    };
    int32_t last_wait = 0;   // the tile of the latest wait (a timeout drains from here)
    auto wait = [&](int32_t c) -> bool {
        last_wait = c;
        const bool ok = hsdev::mbar_wait_bounded(bars + (c & (STAGES - 1)), (uint32_t)((c / STAGES) & 1));
        return __all_sync(0xffffffffu, ok);
    };
    auto release = [&](int32_t c) {
        __syncwarp();
        if (lane == 0 && c + STAGES < total) {
            hsdev::fence_proxy_async_smem();
            issue(c + STAGES);
        }
    };
    if (lane == 0) {
        for (int s = 0; s < STAGES; ++s) hsdev::mbar_init(bars + s, 1);
        hsdev::fence_barrier_init();
    }
    __syncwarp();
    if (lane == 0)
        for (int32_t c = 0; c < min(total, STAGES); ++c) issue(c);
    __syncwarp();

    int32_t c = 0;
    PrecItem nit{};   // the next item, loaded one item ahead
    if (my_items > 0) nit = items[w0];
    for (int32_t ii = 0; ii < my_items; ++ii) {
        // A converged slot's z is computed too (harmless: the dot and p kernels
        // skip it, its r is frozen) -- no dependent load of its flag here.
        const PrecItem it = nit;
        if (ii + 1 < my_items) nit = items[w0 + (ii + 1) * wstride];
        float d[PS];
#pragma unroll
        for (int li = 0; li < PS; ++li) d[li] = it.Di[(int64_t)li * it.npad + lane];
        // r of the rows this lane moves (kept for the fused r.z when it fits in registers)
        constexpr int KR = PS <= 16 ? PS : 1;
        double rkeep[KR];
#pragma unroll
        for (int m = 0; m < PS; ++m) {
            const int t = lane + 32 * m;
            const double rv = t < it.rows ? it.x[t] : 0.0;
            if (PS <= 16) rkeep[m < KR ? m : 0] = rv;
            xs[(t / PS) * XS + (t % PS)] = (float)rv;
        }
        __syncwarp();
        float yv[PS];
#pragma unroll
        for (int li = 0; li < PS; ++li) yv[li] = xs[lane * XS + li];
#pragma unroll
        for (int li = 0; li < PS; ++li) {
            float acc = 0.0f;
#pragma unroll
            for (int lj = 0; lj < li; ++lj) {
                const int e = li * (li - 1) / 2 + lj;
                if (e % E == 0 && !wait(c + e / E)) goto timeout;
                acc = __fadd_rn(acc, __fmul_rn(ring[((c + e / E) & (STAGES - 1)) * (E * 32) + (e % E) * 32 + lane],
                                               yv[lj]));
                if (e % E == E - 1 || e == TLEN - 1) release(c + e / E);
            }
            yv[li] = __fdiv_rn(__fsub_rn(yv[li], acc), d[li]);
        }
        c += NT;
#pragma unroll
        for (int li = 0; li < PS; ++li) yv[li] = __fmul_rn(d[li], yv[li]);
#pragma unroll
        for (int li = PS - 1; li >= 0; --li) {
            float acc = 0.0f;
#pragma unroll
            for (int lj = li + 1; lj < PS; ++lj) {
                const int q = PS - 1 - li;
                const int e = q * (q - 1) / 2 + (lj - li - 1);
                if (e % E == 0 && !wait(c + e / E)) goto timeout;
                acc = __fadd_rn(acc, __fmul_rn(ring[((c + e / E) & (STAGES - 1)) * (E * 32) + (e % E) * 32 + lane],
                                               yv[lj]));
                if (e % E == E - 1 || e == TLEN - 1) release(c + e / E);
            }
            yv[li] = __fdiv_rn(__fsub_rn(yv[li], acc), d[li]);
        }
        c += NT;
        __syncwarp();
#pragma unroll
        for (int li = 0; li < PS; ++li) xs[lane * XS + li] = yv[li];
        __syncwarp();
        hsdev::DD part{0.0, 0.0};   // this item's share of r.z (fused: no separate pass)
#pragma unroll
        for (int m = 0; m < PS; ++m) {
            const int t = lane + 32 * m;
            if (t < it.rows) {
                const double z = (double)xs[(t / PS) * XS + (t % PS)];
                it.y[t] = z;
                hsdev::dd_add_prod(part, PS <= 16 ? rkeep[m < KR ? m : 0] : it.x[t], z);
            }
        }
        part = hsdev::warp_dd(part);
        if (lane == 0) {
            const int64_t item = w0 + (int64_t)ii * wstride;
            rz_part[2 * item] = part.s;
            rz_part[2 * item + 1] = part.c;
        }
        __syncwarp();
    }
    return;
timeout:
    if (lane == 0) hsdev::report_error(err, hsdev::kErrWaitTimeout);
    {
        const int32_t end = min(total, last_wait + STAGES);
        for (int32_t cc = last_wait; cc < end; ++cc)
            (void)hsdev::mbar_wait_bounded(bars + (cc & (STAGES - 1)), (uint32_t)((cc / STAGES) & 1));
    }
}

template <int PS>
constexpr uint32_t batched_warp_bytes() {
    return ((16 * 32 * 4 * 4) + 8 * 4 + 32 * (PS + 1) * 4 + 127) / 128 * 128;
}

// ---- persistent schedule: every iteration of every slot in one launch -----
// The work of a batched iteration is cut into CTA-sized items, ordered by
// (iteration, phase, slot, chunk), with the phases
//   0  q = A p and p.q partials            one item per kPairs chunks of kRPC rows
//   1  x += alpha p, r -= alpha q, r.r     likewise
//   2  z = M^-1 r and r.z partials         one item per kPW * kGPW groups
//   3  p = z + beta p                      one item per kPairs chunks
// CTAs take kTake consecutive items per ticket from one counter.  The first
// item of a slot's phase (its closer) waits until the slot's previous phase is
// open and every item of it has been counted, computes that phase's scalar (alpha before
// phase 1, the convergence test before 2, beta before 3) with the segmented
// kernels' fixed-order reductions -- the iterates are bitwise those of the
// segmented schedule -- and publishes the slot's stage, which the phase's
// other items wait for.  Every wait is for items earlier in the order, taken
// by running CTAs that never wait for a later item, so a launch cannot
// deadlock however many CTAs are resident.  A finished item is counted with a
// fire-and-forget atomic.  Waits poll for at most kStageWaitNs; one that runs
// out sets the abort word and the launch ends with HS_ERR_TIMEOUT.
// One kernel holds the registers and shared memory of its largest phase for
// all phases (2 CTAs of 256 threads per SM), so an item carries two chunks
// (phase 2: two groups per warp) whose loads are interleaved: the
// latency-bound SpMV gets its memory parallelism per warp instead of from
// more warps.  The phase bodies are separate (non-inlined) functions, each
// with the kernel's 128 registers to itself (inlined together they spilled).
constexpr int kPW = kT / 32;   // warps per CTA
constexpr int kPairs = 2;      // chunks per item (phases 0, 1, 3)
constexpr int kGPW = 2;        // groups per warp per item (phase 2)
constexpr int kTake = 4;       // items per ticket
constexpr int32_t kStageDone = 1 << 30;
constexpr uint64_t kStageWaitNs = 2000000000ull;
constexpr uint32_t kPWarpBytes = batched_warp_bytes<32>();   // per-warp ring + staging, largest partsize

struct Work {
    int32_t slot;     // slot index (SlotDev, Scalars, stage words)
    int16_t phase;    // 0..3 as above
    int16_t closer;   // the slot's first item of this phase
    int32_t first;    // phases 0, 1, 3: first BlockMap entry; phase 2: first PrecItem
    int32_t count;    // chunks (phases 0, 1, 3) or groups (phase 2) in the item
};

// Control words: [0] ticket, [1] CTAs that left, [2] abort, [3] unused, then
// per slot s: [4 + 2 s] stage (4 t + phase that may run, or kStageDone),
// [5 + 2 s] items of the current phase finished.
constexpr int kCtl = 4;

__device__ __forceinline__ int32_t phase_items(const SlotDev& sd, int ph) {
    return ph == 2 ? (sd.nitems + kPW * kGPW - 1) / (kPW * kGPW) : (sd.nblk + kPairs - 1) / kPairs;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Thread 0, bounded poll.  Other items: until the stage reaches `need`.
// Closer: until the previous phase is open (stage need - 1: the counter holds
// that phase's items, not the phase before it) and its `nprev` items are
// counted.  Returns 0 (go), 1 (the slot has finished: skip) or 2 (abort).
// The fence after the observed words orders the CTA's later loads (after the
// caller's __syncthreads) behind the writes of the CTAs that published them.
__device__ __forceinline__ int wait_slot(const int32_t* stw, bool closer, int32_t need, int32_t nprev,
                                         int32_t* abortw, int32_t* err) {
    const volatile int32_t* vst = stw;
    const volatile int32_t* vfin = stw + 1;
    const volatile int32_t* vab = abortw;
    uint64_t t0 = 0;
    for (uint32_t k = 0;; ++k) {
        const int32_t v = *vst;
        if (v >= kStageDone) {
            __threadfence();
            return 1;
        }
        if (closer ? (v >= need - 1 && *vfin >= nprev) : v >= need) {
            __threadfence();
            return 0;
        }
        if (*vab) return 2;
        if (k == 0) t0 = globaltimer_ns();
        if ((k & 15) == 15 && globaltimer_ns() - t0 > kStageWaitNs) {
            atomicExch(abortw, 1);
            hsdev::report_error(err, hsdev::kErrWaitTimeout);
            return 2;
        }
        __nanosleep(64);
    }
}

__device__ __forceinline__ void store_dd_at(double* partials, int32_t idx, DD v) {
    v = hsdev::block_dd(v);
    if (threadIdx.x == 0) {
        partials[2 * idx] = v.s;
        partials[2 * idx + 1] = v.c;
    }
}

// range_sum over partials written in this launch: L2 loads (no stale L1 or
// read-only-cache copies), same order as range_sum.
__device__ __noinline__ double range_sum_l2(const double* partials, int32_t first, int32_t count) {
    DD v{0.0, 0.0};
    const double2* p2 = reinterpret_cast<const double2*>(partials) + first;
    for (int base = threadIdx.x; base < count; base += 8 * blockDim.x) {
        double2 w[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (base + k * (int)blockDim.x < count) w[k] = __ldcg(p2 + base + k * blockDim.x);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (base + k * (int)blockDim.x < count) v = hsdev::dd_add(v, DD{w[k].x, w[k].y});
    }
    return hsdev::dd_value(hsdev::block_dd(v));
}

// Phase 0 over `count` chunks of one slot (seg_spmv_dot's arithmetic per
// chunk): the two chunks' 32-row slices are folded side by side, so a warp
// keeps two dependent load chains in flight.
__device__ __noinline__ void pers_spmv(const BlockMap* __restrict__ mm, int count, double* partials, int32_t idx) {
    constexpr int NS = kRPC / kT;
    constexpr int KU = 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const BlockMap ma = mm[0];
    const BlockMap mb = mm[count > 1 ? 1 : 0];
    const int64_t nsl = ((int64_t)ma.n + 31) / 32;
    int64_t oa0[NS], oa1[NS], ob0[NS], ob1[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const int64_t sa = ((int64_t)ma.row0 >> 5) + k * kPW + warp;
        const int64_t sb = ((int64_t)mb.row0 >> 5) + k * kPW + warp;
        oa0[k] = sa < nsl ? __ldg(ma.soff + sa) : 0;
        oa1[k] = sa < nsl ? __ldg(ma.soff + sa + 1) : 0;
        ob0[k] = count > 1 && sb < nsl ? __ldg(mb.soff + sb) : 0;
        ob1[k] = count > 1 && sb < nsl ? __ldg(mb.soff + sb + 1) : 0;
    }
    const double* p = ma.p;   // written in this launch: plain loads
    DD pa{0.0, 0.0}, pb{0.0, 0.0};
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const int64_t ra0 = (int64_t)ma.row0 + (k * kPW + warp) * 32;
        const int64_t rb0 = (int64_t)mb.row0 + (k * kPW + warp) * 32;
        const bool va = ra0 < ma.n, vb = count > 1 && rb0 < mb.n;
        if (!va && !vb) break;   // uniform over the warp
        const int32_t wa = va ? (int32_t)((oa1[k] - oa0[k]) / 32) : 0;
        const int32_t wb = vb ? (int32_t)((ob1[k] - ob0[k]) / 32) : 0;
        const int32_t* __restrict__ cpa = ma.scol + oa0[k] + lane;
        const double* __restrict__ vpa = ma.sval + oa0[k] + lane;
        const int32_t* __restrict__ cpb = mb.scol + ob0[k] + lane;
        const double* __restrict__ vpb = mb.sval + ob0[k] + lane;
        double acca = 0.0, accb = 0.0;
        const int32_t w = wa > wb ? wa : wb;
        for (int32_t j = 0; j < w; j += KU) {   // slice_row_fold's order, per slice
            int32_t ca[KU], cb[KU];
            double aa[KU], ab[KU], xa[KU], xb[KU];
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                ca[u] = j + u < wa ? __ldg(cpa + 32 * (j + u)) : -1;
                aa[u] = j + u < wa ? __ldg(vpa + 32 * (j + u)) : 0.0;
                cb[u] = j + u < wb ? __ldg(cpb + 32 * (j + u)) : -1;
                ab[u] = j + u < wb ? __ldg(vpb + 32 * (j + u)) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                xa[u] = ca[u] >= 0 ? p[ca[u]] : 0.0;
                xb[u] = cb[u] >= 0 ? p[cb[u]] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                if (ca[u] >= 0) acca = __dadd_rn(acca, __dmul_rn(aa[u], xa[u]));
                if (cb[u] >= 0) accb = __dadd_rn(accb, __dmul_rn(ab[u], xb[u]));
            }
        }
        const int64_t ra = ra0 + lane, rb = rb0 + lane;
        if (va && ra < ma.n) {
            ma.q[ra] = acca;
            hsdev::dd_add_prod(pa, p[ra], acca);
        }
        if (vb && rb < mb.n) {
            mb.q[rb] = accb;
            hsdev::dd_add_prod(pb, p[rb], accb);
        }
    }
    store_dd_at(partials, idx, pa);
    if (count > 1) store_dd_at(partials, idx + 1, pb);
}

// Phase 1 over `count` chunks (seg_update's arithmetic per chunk).
__device__ __noinline__ void pers_update(const BlockMap* __restrict__ mm, int count, double alpha, double* partials,
                                         int32_t idx) {
    BlockMap m[kPairs];
    double xv[kPairs][kSub], pv[kPairs][kSub], rv[kPairs][kSub], qv[kPairs][kSub];
#pragma unroll
    for (int c = 0; c < kPairs; ++c) {
        m[c] = mm[c < count ? c : 0];
#pragma unroll
        for (int k = 0; k < kSub; ++k) {
            const int i = m[c].row0 + k * kRPB + threadIdx.x;
            if (c < count && i < m[c].n) {
                xv[c][k] = m[c].x[i];
                pv[c][k] = m[c].p[i];
                rv[c][k] = m[c].r[i];
                qv[c][k] = m[c].q[i];
            }
        }
    }
#pragma unroll
    for (int c = 0; c < kPairs; ++c) {
        if (c >= count) break;   // uniform
        DD part{0.0, 0.0};
#pragma unroll
        for (int k = 0; k < kSub; ++k) {
            const int i = m[c].row0 + k * kRPB + threadIdx.x;
            if (i < m[c].n) {
                m[c].x[i] = __dadd_rn(xv[c][k], __dmul_rn(alpha, pv[c][k]));
                const double ri = __dsub_rn(rv[c][k], __dmul_rn(alpha, qv[c][k]));
                m[c].r[i] = ri;
                hsdev::dd_add_prod(part, ri, ri);
            }
        }
        store_dd_at(partials, idx + c, part);
    }
}

// Phase 3 over `count` chunks (seg_p's arithmetic).
__device__ __noinline__ void pers_p(const BlockMap* __restrict__ mm, int count, double beta) {
    BlockMap m[kPairs];
    double zv[kPairs][kSub], pv[kPairs][kSub];
#pragma unroll
    for (int c = 0; c < kPairs; ++c) {
        m[c] = mm[c < count ? c : 0];
#pragma unroll
        for (int k = 0; k < kSub; ++k) {
            const int i = m[c].row0 + k * kRPB + threadIdx.x;
            if (c < count && i < m[c].n) {
                zv[c][k] = m[c].z[i];
                pv[c][k] = m[c].p[i];
            }
        }
    }
#pragma unroll
    for (int c = 0; c < kPairs; ++c) {
#pragma unroll
        for (int k = 0; k < kSub; ++k) {
            const int i = m[c].row0 + k * kRPB + threadIdx.x;
            if (c < count && i < m[c].n) m[c].p[i] = __dadd_rn(zv[c][k], __dmul_rn(beta, pv[c][k]));
        }
    }
}

// Phase 2 for up to kGPW groups of one warp (l1gs_batched_kernel's
// arithmetic per group), streamed through the warp's ring: the next group's
// first tiles are in flight while the current one is solved.  The ring
// position `c` runs on across items (stage c % 4, parity (c / 4) % 2), so
// every tile is issued and waited for exactly once.  False after a bounded
// wait ran out.
template <int PS>
__device__ __noinline__ bool pers_apply(const PrecItem* __restrict__ items, int64_t g0, int ng, unsigned char* wbase,
                                        uint32_t& c, double* rz_part) {
    constexpr int E = kBatchE;
    constexpr int STAGES = 4;
    constexpr int TLEN = PS * (PS - 1) / 2;
    constexpr int NT = (TLEN + E - 1) / E;
    constexpr uint32_t NTPG = 2 * NT;
    constexpr int XS = PS + 1;
    constexpr uint32_t kRing = E * 32 * 4 * STAGES;
    static_assert(kRing + 8 * STAGES + 32 * XS * 4 <= kPWarpBytes, "per-warp shared memory");
    const int lane = threadIdx.x & 31;
    float* ring = reinterpret_cast<float*>(wbase);
    uint64_t* bars = reinterpret_cast<uint64_t*>(wbase + kRing);
    float* xs = reinterpret_cast<float*>(wbase + kRing + 8 * STAGES);
    const uint32_t c0 = c, end = c0 + (uint32_t)ng * NTPG;
    const float* st0 = items[g0].ST;
    const float* st1 = ng > 1 ? items[g0 + kPW].ST : st0;
    auto issue = [&](uint32_t k) {   // lane 0
        const uint32_t r = k - c0;
        const uint32_t j = r / NTPG;
        const float* src = (j == 0 ? st0 : st1) + (int64_t)(r - j * NTPG) * E * 32;
        const uint32_t s = k & (STAGES - 1);
        hsdev::mbar_arrive_expect_tx(bars + s, (uint32_t)(E * 32 * 4));
        hsdev::bulk_load(ring + s * (E * 32), src, (uint32_t)(E * 32 * 4), bars + s);
    };
    uint32_t last_wait = c0;
    auto wait = [&](uint32_t k) -> bool {
        last_wait = k;
        const bool ok = hsdev::mbar_wait_bounded(bars + (k & (STAGES - 1)), (k / STAGES) & 1u);
        return __all_sync(0xffffffffu, ok);
    };
    auto release = [&](uint32_t k) {
        __syncwarp();
        if (lane == 0 && k + STAGES < end) {
            hsdev::fence_proxy_async_smem();
            issue(k + STAGES);
        }
    };
    // The ring's stages were last read by this warp's previous item.
    __syncwarp();
    if (lane == 0) {
        hsdev::fence_proxy_async_smem();
        for (uint32_t k = c0; k < end && k < c0 + STAGES; ++k) issue(k);
    }
    for (int j = 0; j < ng; ++j) {
        const int64_t gi = g0 + (int64_t)j * kPW;
        const PrecItem it = items[gi];
        const uint32_t cj = c0 + (uint32_t)j * NTPG;
        // D_Dl1 in registers up to partsize 16; above, read at each use (L1)
        constexpr bool kDReg = PS <= 16;
        float d[kDReg ? PS : 1];
        if (kDReg) {
#pragma unroll
            for (int li = 0; li < PS; ++li) d[kDReg ? li : 0] = __ldg(it.Di + (int64_t)li * it.npad + lane);
        }
        auto dl = [&](int li) { return kDReg ? d[kDReg ? li : 0] : __ldg(it.Di + (int64_t)li * it.npad + lane); };
#pragma unroll
        for (int m = 0; m < PS; ++m) {
            const int t = lane + 32 * m;
            xs[(t / PS) * XS + (t % PS)] = t < it.rows ? (float)it.x[t] : 0.0f;
        }
        __syncwarp();
        float yv[PS];
#pragma unroll
        for (int li = 0; li < PS; ++li) yv[li] = xs[lane * XS + li];
#pragma unroll
        for (int li = 0; li < PS; ++li) {
            float acc = 0.0f;
#pragma unroll
            for (int lj = 0; lj < li; ++lj) {
                const int e = li * (li - 1) / 2 + lj;
                const uint32_t k = cj + e / E;
                if (e % E == 0 && !wait(k)) goto timeout;
                acc = __fadd_rn(acc, __fmul_rn(ring[(k & (STAGES - 1)) * (E * 32) + (e % E) * 32 + lane], yv[lj]));
                if (e % E == E - 1 || e == TLEN - 1) release(k);
            }
            yv[li] = __fdiv_rn(__fsub_rn(yv[li], acc), dl(li));
        }
#pragma unroll
        for (int li = 0; li < PS; ++li) yv[li] = __fmul_rn(dl(li), yv[li]);
#pragma unroll
        for (int li = PS - 1; li >= 0; --li) {
            float acc = 0.0f;
#pragma unroll
            for (int lj = li + 1; lj < PS; ++lj) {
                const int q = PS - 1 - li;
                const int e = q * (q - 1) / 2 + (lj - li - 1);
                const uint32_t k = cj + NT + e / E;
                if (e % E == 0 && !wait(k)) goto timeout;
                acc = __fadd_rn(acc, __fmul_rn(ring[(k & (STAGES - 1)) * (E * 32) + (e % E) * 32 + lane], yv[lj]));
                if (e % E == E - 1 || e == TLEN - 1) release(k);
            }
            yv[li] = __fdiv_rn(__fsub_rn(yv[li], acc), dl(li));
        }
        __syncwarp();
#pragma unroll
        for (int li = 0; li < PS; ++li) xs[lane * XS + li] = yv[li];
        __syncwarp();
        DD part{0.0, 0.0};   // this group's share of r.z
#pragma unroll
        for (int m = 0; m < PS; ++m) {
            const int t = lane + 32 * m;
            if (t < it.rows) {
                const double z = (double)xs[(t / PS) * XS + (t % PS)];
                it.y[t] = z;
                hsdev::dd_add_prod(part, it.x[t], z);
            }
        }
        part = hsdev::warp_dd(part);
        if (lane == 0) {
            rz_part[2 * gi] = part.s;
            rz_part[2 * gi + 1] = part.c;
        }
        __syncwarp();
    }
    c = end;
    return true;
timeout:
    // let the copies in flight land before the shared memory is left
    for (uint32_t k = last_wait; k < end && k < last_wait + STAGES; ++k)
        (void)hsdev::mbar_wait_bounded(bars + (k & (STAGES - 1)), (k / STAGES) & 1u);
    c = end;
    return false;
}

__device__ __forceinline__ void reset_stages(int32_t* ctl, const Scalars* scal, const int32_t* active, int32_t nactive,
                                             int first, int stride) {
    for (int32_t a = first; a < nactive; a += stride) {
        const int32_t s = active[a];
        const int done = *reinterpret_cast<const volatile int*>(&scal[s].done);
        ctl[kCtl + 2 * s] = done ? kStageDone : 0;
        ctl[kCtl + 2 * s + 1] = 0;
    }
}

// Before the first launch over a new active set.
__global__ void persist_reset(int32_t* ctl, const Scalars* scal, const int32_t* active, int32_t nactive) {
    if (threadIdx.x == 0) {
        ctl[0] = 0;
        ctl[1] = 0;
    }
    reset_stages(ctl, scal, active, nactive, threadIdx.x, blockDim.x);
}

__global__ void __launch_bounds__(kT, 2)
    batch_persistent_kernel(const Work* __restrict__ work, int32_t nwork, int32_t iters,
                            const SlotDev* __restrict__ slots, const int32_t* __restrict__ active, int32_t nactive,
                            const BlockMap* __restrict__ map, const PrecItem* __restrict__ items, double* partials,
                            double* rz_part, Scalars* scal, int32_t* ctl, int32_t maxit, int32_t* err) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int32_t sh_tk, sh_flag, sh_bad;
    __shared__ double sh_val;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wbase = smem + (size_t)warp * kPWarpBytes;
    if (lane == 0) {
        uint64_t* bars = reinterpret_cast<uint64_t*>(wbase + kBatchE * 32 * 4 * 4);
        for (int s = 0; s < 4; ++s) hsdev::mbar_init(bars + s, 1);
        hsdev::fence_barrier_init();
    }
    if (threadIdx.x == 0) sh_bad = 0;
    __syncthreads();
    uint32_t c = 0;   // this warp's ring position
    int32_t* abortw = ctl + 2;
    const int64_t total = (int64_t)nwork * iters;
    bool stop = false;
    while (!stop) {
        if (threadIdx.x == 0) sh_tk = atomicAdd(ctl, 1);
        __syncthreads();
        const int64_t w0 = (int64_t)sh_tk * kTake;
        if (w0 >= total) break;   // uniform
        const int64_t w1 = w0 + kTake < total ? w0 + kTake : total;
        for (int64_t wi = w0; wi < w1; ++wi) {
            const int32_t t = (int32_t)(wi / nwork);
            const Work wk = work[wi - (int64_t)t * nwork];
            const int32_t need = 4 * t + wk.phase;
            int32_t* stw = ctl + kCtl + 2 * wk.slot;
            const SlotDev sd = slots[wk.slot];
            // The closer of phase 0 at the launch's first iteration has no
            // previous phase to close (the stage starts at 0).
            const bool closing = wk.closer && !(t == 0 && wk.phase == 0);
            if (threadIdx.x == 0) {
                const int f = wait_slot(stw, closing, need, closing ? phase_items(sd, (wk.phase + 3) & 3) : 0,
                                        abortw, err);
                sh_flag = f;
                if (f == 0 && !closing && (wk.phase == 1 || wk.phase == 3)) {
                    const volatile Scalars* vs = sd.s;
                    sh_val = wk.phase == 1 ? vs->alpha : vs->beta;
                }
            }
            __syncthreads();
            int flag = sh_flag;
            __syncthreads();
            if (flag == 2) {
                stop = true;
                break;
            }
            if (flag == 1) continue;   // the slot has finished
            if (closing) {
                // the previous phase's scalar, then the stage of this phase
                double v = 0.0;
                if (wk.phase == 1 || wk.phase == 2) v = range_sum_l2(partials, sd.blk0, sd.nblk);
                else if (wk.phase == 3) v = range_sum_l2(rz_part, sd.item0, sd.nitems);
                if (threadIdx.x == 0) {
                    volatile Scalars* vs = sd.s;
                    int32_t next = need;
                    if (wk.phase == 1) {
                        const double a = __ddiv_rn(vs->rz, v);
                        vs->pq = v;
                        vs->alpha = a;
                        sh_val = a;
                    } else if (wk.phase == 2) {
                        const int32_t itn = vs->it + 1;
                        vs->it = itn;
                        vs->rr = v;
                        if (sqrt(v) <= __dmul_rn(vs->rtol, sqrt(vs->bb))) {
                            vs->done = 1;
                            vs->conv_it = itn;
                            next = kStageDone;
                        } else if (itn >= maxit) {
                            vs->done = 2;   // gave up
                            vs->conv_it = itn;
                            next = kStageDone;
                        }
                    } else if (wk.phase == 3) {
                        const double bt = __ddiv_rn(v, vs->rz);
                        vs->beta = bt;
                        vs->rz = v;
                        sh_val = bt;
                    }
                    *reinterpret_cast<volatile int32_t*>(stw + 1) = 0;
                    __threadfence();
                    *reinterpret_cast<volatile int32_t*>(stw) = next;
                    sh_flag = next >= kStageDone ? 1 : 0;
                }
                __syncthreads();
                flag = sh_flag;
                __syncthreads();
                if (flag) continue;   // converged (or stopped) at this check
            }
            const double val = sh_val;
            switch (wk.phase) {
                case 0: pers_spmv(map + wk.first, wk.count, partials, wk.first); break;
                case 1: pers_update(map + wk.first, wk.count, val, partials, wk.first); break;
                case 2:
                    if (warp < wk.count) {
                        const int ng = warp + kPW < wk.count ? 2 : 1;
                        const int64_t g0 = (int64_t)wk.first + warp;
                        bool ok = true;
                        if (sd.ps == 8) ok = pers_apply<8>(items, g0, ng, wbase, c, rz_part);
                        else if (sd.ps == 16) ok = pers_apply<16>(items, g0, ng, wbase, c, rz_part);
                        else ok = pers_apply<32>(items, g0, ng, wbase, c, rz_part);
                        if (!ok && lane == 0) {
                            sh_bad = 1;
                            atomicExch(abortw, 1);
                        }
                    }
                    break;
                default: pers_p(map + wk.first, wk.count, val); break;
            }
            // count the item (no wait for the result)
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(stw + 1, 1);
            }
            if (sh_bad) {   // written before the barrier above
                stop = true;
                break;
            }
        }
        __syncthreads();   // sh_tk is rewritten by the next ticket
    }
    // The last CTA to leave resets the counters for the next launch.
    __syncthreads();
    if (threadIdx.x == 0) {
        if (sh_bad) {
            atomicExch(abortw, 1);
            hsdev::report_error(err, hsdev::kErrWaitTimeout);
        }
        __threadfence();
        const int32_t prev = atomicAdd(ctl + 1, 1);
        if (prev == (int32_t)gridDim.x - 1) {
            __threadfence();
            reset_stages(ctl, scal, active, nactive, 0, 1);
            ctl[0] = 0;
            ctl[1] = 0;
            __threadfence();
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host engine
// ---------------------------------------------------------------------------
struct hs_batch_slot {
    int state = 0;           // 0 free, 1 active, 2 finished (waiting for poll)
    int64_t tag = 0;
    hs_matrix* A = nullptr;
    hs_l1gs* P = nullptr;
    int32_t n = 0, ps = 0;
    double* vec = nullptr;   // x r z p q b (6n doubles)
    float* tiles = nullptr;  // per group: the smoother's tiles, contiguous (batch_tiles_kernel)
    int64_t* soff = nullptr; // the matrix in 32-row slices (slice_fill_kernel)
    int32_t* scol = nullptr;
    double* sval = nullptr;
    double* x_out = nullptr; // host destination
    int64_t bytes = 0;
    int32_t blk0 = 0, nblk = 0;
    bool launched = false;   // part of the active set of the launch in flight
};

struct hs_batch_s {
    hs_batch_config cfg;
    cudaStream_t solve = nullptr, setup = nullptr;
    std::vector<hs_batch_slot> slots;
    SlotDev* d_slots = nullptr;
    Scalars* d_scal = nullptr;
    Scalars* h_scal = nullptr;          // pinned mirror of d_scal
    cudaEvent_t launched = nullptr;     // end of the last hs_batch_launch
    cudaEvent_t admitted = nullptr;     // end of the last admission's setup work
    bool inflight = false;
    bool pending_admission = false;
    BlockMap* d_map = nullptr;
    int32_t* d_active = nullptr;
    PrecItem* d_items = nullptr;
    double* d_partials = nullptr;
    double* d_rzpart = nullptr;   // r.z partials, one pair per L1GS work item
    double* d_init = nullptr;    // init partials (2 x 2 x kRedMaxBlocks)
    int32_t max_blocks = 0, max_items = 0;
    int64_t used = 0;
    // current launch geometry
    int32_t nblocks = 0, nactive = 0;
    struct Cls {
        int ps;
        int32_t item0, nitems;
    };
    std::vector<Cls> classes;
    bool dirty = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int32_t exec_iters = 0;       // iterations in the captured persistent launch
    int32_t* err = nullptr;
    int64_t iterations_run = 0;
    // persistent schedule (cfg.schedule == HS_BATCH_PERSISTENT)
    Work* d_work = nullptr;
    int32_t max_work = 0, nwork = 0, pers_grid = 0;
    int32_t* d_ctl = nullptr;     // ticket, exits, abort, stage words
    int32_t* h_ctl = nullptr;     // pinned copy of the abort word after a launch
};

namespace {

// The slot's matrix in 32-row slices: widths and offsets from the host row
// pointers, entries gathered from the slot's device CSR on the admission
// stream (stream-ordered allocations, no host wait).
int build_slices(hs_batch_slot& sl, int32_t n, const int32_t* rp_host, cudaStream_t st) {
    const int32_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const void* mv = nullptr;
    int mdt = 0;
    hs::matrix_arrays(sl.A, &rp, &ci, &mv, &mdt);
    const int64_t nsl = ((int64_t)n + 31) / 32;
    std::vector<int64_t> off((size_t)nsl + 1);
    int64_t total = 0;
    for (int64_t k = 0; k < nsl; ++k) {
        off[(size_t)k] = total;
        int32_t w = 0;
        const int64_t r1 = std::min<int64_t>((k + 1) * 32, n);
        for (int64_t r = k * 32; r < r1; ++r) w = std::max(w, rp_host[r + 1] - rp_host[r]);
        total += 32 * (int64_t)w;
    }
    off[(size_t)nsl] = total;
    cudaError_t e;
    if ((e = cudaMallocAsync(&sl.soff, sizeof(int64_t) * (size_t)(nsl + 1), st)) ||
        (e = cudaMallocAsync(&sl.scol, sizeof(int32_t) * (size_t)std::max<int64_t>(total, 32), st)) ||
        (e = cudaMallocAsync(&sl.sval, sizeof(double) * (size_t)std::max<int64_t>(total, 32), st)))
        return hs::cuda_error(e, "cudaMallocAsync (slices)");
    // (pageable source: the call returns once the bytes are staged)
    if ((e = cudaMemcpyAsync(sl.soff, off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice, st)))
        return hs::cuda_error(e, "slice offsets");
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((32 * nsl + kT - 1) / kT, 8192));
    hsdev::slice_fill_kernel<double><<<grid, kT, 0, st>>>(n, nsl, rp, ci, static_cast<const double*>(mv), sl.soff, sl.scol, sl.sval);
    hs::count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return hs::cuda_error(e, "slice_fill_kernel");
    return HS_OK;
}

int64_t slot_estimate(int32_t n, int64_t nnz, int ps) {
    const int64_t nparts = (n + ps - 1) / ps;
    const int64_t npad = (nparts + 31) / 32 * 32;
    const int64_t tlen = (int64_t)ps * (ps - 1) / 2;
    const int64_t ntile = (tlen + kBatchE - 1) / kBatchE;
    const int64_t prec = 4 * (2 * tlen * npad + (int64_t)ps * npad + n) + 4 * 2 * ntile * kBatchE * npad;
    const int64_t nsl = ((int64_t)n + 31) / 32;
    const int64_t mat = 4 * (n + 1) + 12 * nnz + 8 * (nsl + 1) + 12 * (nnz + (int64_t)n);   // CSR + slices
    return prec + mat + 6 * 8 * (int64_t)n + 64 * 1024;
}

template <int PS>
int launch_batched(hs_batch* B, const hs_batch_s::Cls& cl, cudaStream_t st) {
    constexpr uint32_t wb = batched_warp_bytes<PS>();
    const int wpb = 4;
    const size_t smem = (size_t)wb * wpb;
    auto kern = l1gs_batched_kernel<PS, kBatchE, 4>;
    if (int rc = hs::ensure_dynamic_smem((const void*)kern, (int)smem)) return rc;
    int per_sm = 0;
    HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpb * 32, smem));
    const int64_t want = (cl.nitems + wpb - 1) / wpb;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)std::max(1, per_sm) * hs::num_sms()));
    kern<<<grid, wpb * 32, smem, st>>>(B->d_items + cl.item0, cl.nitems, B->d_rzpart + 2 * (size_t)cl.item0, B->err);
    HS_LAUNCH_CHECK("l1gs_batched_kernel");
    return HS_OK;
}

int launch_prec_class(hs_batch* B, const hs_batch_s::Cls& cl, cudaStream_t st) {
    switch (cl.ps) {
        case 8: return launch_batched<8>(B, cl, st);
        case 16: return launch_batched<16>(B, cl, st);
        case 32: return launch_batched<32>(B, cl, st);
        default: return hs::set_error(HS_ERR_UNSUPPORTED, "batched partsize %d", cl.ps);
    }
}

// Rebuild the device tables for the current active set.
int rebuild(hs_batch* B) {
    std::vector<BlockMap> map;
    std::vector<int32_t> active;
    std::vector<PrecItem> items;
    B->classes.clear();
    std::vector<int32_t> item0(B->slots.size(), 0), nitem(B->slots.size(), 0);
    for (int ps : {8, 16, 32}) {
        hs_batch_s::Cls cl{ps, (int32_t)items.size(), 0};
        for (size_t s = 0; s < B->slots.size(); ++s) {
            const hs_batch_slot& sl = B->slots[s];
            if (sl.state != 1 || sl.ps != ps) continue;
            item0[s] = (int32_t)items.size();
            hs::L1gsView lv;
            hs::l1gs_view_of(sl.P, &lv);
            const double* r = sl.vec + sl.n;
            double* z = sl.vec + 2 * (size_t)sl.n;
            for (int32_t g = 0; g < lv.ngroups; ++g) {
                PrecItem it{};
                it.ST = sl.tiles + (int64_t)g * 2 * ((lv.tlen + kBatchE - 1) / kBatchE) * kBatchE * 32;
                it.Di = static_cast<const float*>(lv.Di) + (int64_t)g * 32;
                const int64_t row0 = (int64_t)g * 32 * ps;
                it.x = r + row0;
                it.y = z + row0;
                it.npad = lv.npad;
                it.rows = (int32_t)std::max<int64_t>(0, (int64_t)sl.n - row0);
                it.tlen = lv.tlen;
                it.s = B->d_scal + s;
                items.push_back(it);
            }
            nitem[s] = (int32_t)items.size() - item0[s];
        }
        cl.nitems = (int32_t)items.size() - cl.item0;
        if (cl.nitems) B->classes.push_back(cl);
    }
    std::vector<SlotDev> sd(B->slots.size());
    for (size_t s = 0; s < B->slots.size(); ++s) {
        hs_batch_slot& sl = B->slots[s];
        if (sl.state != 1) continue;
        active.push_back((int32_t)s);
        sl.blk0 = (int32_t)map.size();
        sl.nblk = (sl.n + kRPC - 1) / kRPC;
        BlockMap m{};
        m.soff = sl.soff;
        m.scol = sl.scol;
        m.sval = sl.sval;
        m.n = sl.n;
        m.x = sl.vec;
        m.r = sl.vec + sl.n;
        m.z = sl.vec + 2 * (size_t)sl.n;
        m.p = sl.vec + 3 * (size_t)sl.n;
        m.q = sl.vec + 4 * (size_t)sl.n;
        m.s = B->d_scal + s;
        for (int32_t b = 0; b < sl.nblk; ++b) {
            m.row0 = b * kRPC;
            map.push_back(m);
        }
        sd[s] = SlotDev{sl.n, sl.blk0, sl.nblk, item0[s], nitem[s], sl.ps, B->d_scal + s};
    }
    // Persistent schedule: one iteration's work items in (phase, slot, chunk) order.
    std::vector<Work> work;
    if (B->cfg.schedule == HS_BATCH_PERSISTENT) {
        for (int32_t ph = 0; ph < 4; ++ph)
            for (int32_t s : active) {
                const hs_batch_slot& sl = B->slots[(size_t)s];
                if (ph == 2) {
                    for (int32_t g = 0; g < nitem[(size_t)s]; g += kPW * kGPW)
                        work.push_back(Work{s, 2, (int16_t)(g == 0), item0[(size_t)s] + g,
                                            std::min<int32_t>(kPW * kGPW, nitem[(size_t)s] - g)});
                } else {
                    for (int32_t b = 0; b < sl.nblk; b += kPairs)
                        work.push_back(Work{s, (int16_t)ph, (int16_t)(b == 0), sl.blk0 + b,
                                            std::min<int32_t>(kPairs, sl.nblk - b)});
                }
            }
        if ((int32_t)work.size() > B->max_work) {
            cudaFree(B->d_work);
            B->d_work = nullptr;
            B->max_work = std::max<int32_t>((int32_t)work.size() * 2, 4096);
            HS_CUDA(cudaMalloc(&B->d_work, sizeof(Work) * B->max_work));
        }
    }
    if ((int32_t)map.size() > B->max_blocks || (int32_t)items.size() > B->max_items) {
        cudaFree(B->d_map);
        cudaFree(B->d_partials);
        cudaFree(B->d_items);
        cudaFree(B->d_rzpart);
        B->max_blocks = std::max<int32_t>((int32_t)map.size() * 2, 1024);
        B->max_items = std::max<int32_t>((int32_t)items.size() * 2, 1024);
        HS_CUDA(cudaMalloc(&B->d_map, sizeof(BlockMap) * B->max_blocks));
        HS_CUDA(cudaMalloc(&B->d_partials, 2 * sizeof(double) * B->max_blocks));
        HS_CUDA(cudaMalloc(&B->d_items, sizeof(PrecItem) * B->max_items));
        HS_CUDA(cudaMalloc(&B->d_rzpart, 2 * sizeof(double) * B->max_items));
    }
    cudaStream_t st = B->solve;
    if (!sd.empty())
        HS_CUDA(cudaMemcpyAsync(B->d_slots, sd.data(), sizeof(SlotDev) * sd.size(), cudaMemcpyHostToDevice, st));
    if (!map.empty()) HS_CUDA(cudaMemcpyAsync(B->d_map, map.data(), sizeof(BlockMap) * map.size(), cudaMemcpyHostToDevice, st));
    if (!active.empty())
        HS_CUDA(cudaMemcpyAsync(B->d_active, active.data(), sizeof(int32_t) * active.size(), cudaMemcpyHostToDevice, st));
    if (!items.empty())
        HS_CUDA(cudaMemcpyAsync(B->d_items, items.data(), sizeof(PrecItem) * items.size(), cudaMemcpyHostToDevice, st));
    if (!work.empty()) {
        HS_CUDA(cudaMemcpyAsync(B->d_work, work.data(), sizeof(Work) * work.size(), cudaMemcpyHostToDevice, st));
        persist_reset<<<1, kT, 0, st>>>(B->d_ctl, B->d_scal, B->d_active, (int32_t)active.size());
        hs::count_launch();
        HS_CUDA(cudaGetLastError());
    }
    HS_CUDA(cudaStreamSynchronize(st));   // host vectors above go out of scope
    B->nblocks = (int32_t)map.size();
    B->nactive = (int32_t)active.size();
    B->nwork = (int32_t)work.size();
    if (B->exec) {
        cudaGraphExecDestroy(B->exec);
        B->exec = nullptr;
    }
    if (B->graph) {
        cudaGraphDestroy(B->graph);
        B->graph = nullptr;
    }
    B->dirty = false;
    return HS_OK;
}

// The persistent kernel's shared memory and resident CTAs (before any capture).
int prepare_persistent(hs_batch* B) {
    const size_t smem = (size_t)kPW * kPWarpBytes;
    if (int rc = hs::ensure_dynamic_smem((const void*)batch_persistent_kernel, (int)smem)) return rc;
    if (!B->pers_grid) {
        int per_sm = 0;
        HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_persistent_kernel, kT, smem));
        B->pers_grid = std::max(1, per_sm) * hs::num_sms();
    }
    return HS_OK;
}

// `iters` iterations of every active slot: one persistent launch (several only
// when the ticket count would pass 2^30).
int enqueue_persistent(hs_batch* B, int32_t iters, cudaStream_t st) {
    const size_t smem = (size_t)kPW * kPWarpBytes;
    const int32_t kmax = (int32_t)std::max<int64_t>(1, ((int64_t)1 << 30) / std::max<int32_t>(B->nwork, 1));
    for (int32_t done = 0; done < iters;) {
        const int32_t k = std::min(iters - done, kmax);
        const int64_t tickets = ((int64_t)B->nwork * k + kTake - 1) / kTake;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tickets, B->pers_grid));
        batch_persistent_kernel<<<grid, kT, smem, st>>>(B->d_work, B->nwork, k, B->d_slots, B->d_active, B->nactive,
                                                       B->d_map, B->d_items, B->d_partials, B->d_rzpart, B->d_scal,
                                                       B->d_ctl, B->cfg.maxit, B->err);
        hs::count_launch();
        HS_LAUNCH_CHECK("batch_persistent_kernel");
        done += k;
    }
    return HS_OK;
}

int enqueue_iteration(hs_batch* B, cudaStream_t st) {
    if (B->nactive == 0) return HS_OK;
    seg_spmv_dot<<<B->nblocks, kT, 0, st>>>(B->d_map, B->d_partials);
    seg_alpha<<<B->nactive, kT, 0, st>>>(B->d_slots, B->d_active, B->d_partials);
    seg_update<<<B->nblocks, kT, 0, st>>>(B->d_map, B->d_partials);
    seg_check<<<B->nactive, kT, 0, st>>>(B->d_slots, B->d_active, B->d_partials, B->cfg.maxit);
    hs::count_launch(4);
    for (const auto& cl : B->classes) {
        int rc = launch_prec_class(B, cl, st);
        if (rc) return rc;
    }
    seg_beta<<<B->nactive, kT, 0, st>>>(B->d_slots, B->d_active, B->d_rzpart);
    seg_p<<<B->nblocks, kT, 0, st>>>(B->d_map);
    hs::count_launch(2);
    HS_CUDA(cudaGetLastError());
    return HS_OK;
}

// Stream-ordered release on the solve stream: after every launch that used
// the slot, without waiting for the device.
void free_slot(hs_batch* B, hs_batch_slot& sl) {
    if (sl.P) hs::l1gs_destroy_async(sl.P, B->solve);
    if (sl.A) hs::matrix_destroy_async(sl.A, B->solve);
    if (sl.vec) cudaFreeAsync(sl.vec, B->solve);
    if (sl.tiles) cudaFreeAsync(sl.tiles, B->solve);
    if (sl.soff) cudaFreeAsync(sl.soff, B->solve);
    if (sl.scol) cudaFreeAsync(sl.scol, B->solve);
    if (sl.sval) cudaFreeAsync(sl.sval, B->solve);
    B->used -= sl.bytes;
    sl = hs_batch_slot();
}

}  // namespace

namespace {
// Admission runs while the solve graph occupies the GPU: give its stream the
// highest priority so its (small) setup kernels are scheduled ahead of the
// queued iteration blocks instead of behind them.
cudaError_t create_setup_stream(cudaStream_t* st) {
    int lo = 0, hi = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (e != cudaSuccess) return e;
    return cudaStreamCreateWithPriority(st, cudaStreamNonBlocking, hi);
}
}  // namespace

extern "C" {

int hs_batch_create(const hs_batch_config* cfg, void* stream, hs_batch** out) {
    (void)stream;
    if (!cfg || !out) return hs::set_error(HS_ERR_ARG, "hs_batch_create: NULL argument");
    *out = nullptr;
    if (cfg->max_slots < 1 || cfg->max_slots > 4096) return hs::set_error(HS_ERR_ARG, "max_slots out of range");
    if (cfg->hbm_budget <= 0) return hs::set_error(HS_ERR_ARG, "hbm_budget must be positive");
    if (cfg->maxit < 1) return hs::set_error(HS_ERR_ARG, "maxit must be positive");
    if (cfg->schedule != HS_BATCH_PERSISTENT && cfg->schedule != HS_BATCH_SEGMENTED)
        return hs::set_error(HS_ERR_ARG, "schedule must be HS_BATCH_PERSISTENT or HS_BATCH_SEGMENTED");
    hs_batch* B = new hs_batch();
    B->cfg = *cfg;
    B->slots.resize(cfg->max_slots);
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&B->solve, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&B->launched, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&B->admitted, cudaEventDisableTiming)) ||
        (e = cudaMallocHost(&B->h_scal, sizeof(Scalars) * cfg->max_slots)) ||
        (e = create_setup_stream(&B->setup)) ||
        (e = cudaMalloc(&B->d_slots, sizeof(SlotDev) * cfg->max_slots)) ||
        (e = cudaMalloc(&B->d_scal, sizeof(Scalars) * cfg->max_slots)) ||
        (e = cudaMalloc(&B->d_active, sizeof(int32_t) * cfg->max_slots)) ||
        (e = cudaMalloc(&B->d_init, sizeof(double) * 4 * hsdev::kRedMaxBlocks)) ||
        (e = cudaMalloc(&B->d_ctl, sizeof(int32_t) * (kCtl + 2 * (size_t)cfg->max_slots))) ||
        (e = cudaMallocHost(&B->h_ctl, sizeof(int32_t)))) {
        hs_batch_destroy(B);
        return hs::cuda_error(e, "hs_batch_create");
    }
    B->h_ctl[0] = 0;
    cudaMemset(B->d_ctl, 0, sizeof(int32_t) * (kCtl + 2 * (size_t)cfg->max_slots));
    cudaMemset(B->d_scal, 0, sizeof(Scalars) * cfg->max_slots);
    // Reserve the budget (at most 90 % of the free memory) in the stream-ordered
    // pool the slots allocate from, so admissions take memory the pool holds
    // instead of mapping new memory while systems are being solved.
    hs::keep_pool_reserve();
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        const size_t want = (size_t)std::min<int64_t>(cfg->hbm_budget, (int64_t)(0.9 * (double)free_b));
        void* p = nullptr;
        if (want > 0 && cudaMallocAsync(&p, want, B->setup) == cudaSuccess) {
            cudaFreeAsync(p, B->setup);
            cudaStreamSynchronize(B->setup);
        }
        cudaGetLastError();   // a reserve that could not be made is not an error
    }
    B->err = hs::device_error_word();
    *out = B;
    return HS_OK;
}

int hs_batch_submit(hs_batch* B, const hs_sparse* A, const double* b_host, double* x_host, int64_t tag,
                    int32_t partsize, int32_t* slot_out) {
    if (!B || !A || !b_host || !x_host) return hs::set_error(HS_ERR_ARG, "hs_batch_submit: NULL argument");
    const int ps = partsize > 0 ? partsize : B->cfg.partsize;
    if (ps != 8 && ps != 16 && ps != 32) return hs::set_error(HS_ERR_ARG, "batched partsize must be 8, 16 or 32");
    int32_t free_idx = -1;
    for (size_t s = 0; s < B->slots.size(); ++s)
        if (B->slots[s].state == 0) {
            free_idx = (int32_t)s;
            break;
        }
    const int64_t est = slot_estimate(A->n, A->nnz, ps);
    // A request larger than the whole budget can never be admitted: say so
    // (HS_ERR_ARG) instead of "not now" (HS_ERR_BUDGET), so a caller waiting
    // for memory to free up does not wait forever.
    if (est > B->cfg.hbm_budget)
        return hs::set_error(HS_ERR_ARG, "system needs %lld bytes, more than the whole HBM budget %lld",
                             (long long)est, (long long)B->cfg.hbm_budget);
    if (free_idx < 0 || B->used + est > B->cfg.hbm_budget)
        return hs::set_error(HS_ERR_BUDGET, "no free slot or HBM budget (%lld + %lld > %lld)", (long long)B->used,
                             (long long)est, (long long)B->cfg.hbm_budget);
    hs_batch_slot sl;
    sl.tag = tag;
    sl.n = A->n;
    sl.ps = ps;
    sl.x_out = x_host;
    // The engine solves SPD systems (CG): a symmetric CSC's columns are its
    // rows, so the arrays are uploaded once, as CSR, and the FP32 smoother is
    // packed from that device copy (isSymA reads column i as row i).
    // Slot memory is stream-ordered: allocated on the setup stream, released
    // on the solve stream after the slot's last use, with no device sync.
    hs_sparse rows = *A;
    rows.format = HS_CSR;
    int rc = hs::matrix_create_async(&rows, HS_F64, B->setup, &sl.A);
    if (!rc) rc = hs::l1gs_create_from_matrix(sl.A, ps, 1.5, HS_SWEEP_SYMMETRIC, HS_F32, B->setup, &sl.P);
    if (!rc) {
        cudaError_t e = cudaMallocAsync(&sl.vec, sizeof(double) * 6 * (size_t)A->n, B->setup);
        if (e) rc = hs::cuda_error(e, "cudaMallocAsync (slot vectors)");
    }
    if (!rc) rc = build_slices(sl, A->n, A->ptr, B->setup);
    if (!rc) {   // the smoother's tiles, regrouped for the batched kernel
        hs::L1gsView lv;
        hs::l1gs_view_of(sl.P, &lv);
        const int32_t nt = (int32_t)((lv.tlen + kBatchE - 1) / kBatchE);
        const int64_t count = (int64_t)lv.ngroups * 2 * nt * kBatchE * 32;
        cudaError_t e = cudaMallocAsync(&sl.tiles, sizeof(float) * (size_t)std::max<int64_t>(count, 32), B->setup);
        if (e) {
            rc = hs::cuda_error(e, "cudaMallocAsync (slot tiles)");
        } else if (count > 0) {
            const int grid = (int)std::min<int64_t>((count + kT - 1) / kT, 8192);
            batch_tiles_kernel<kBatchE><<<grid, kT, 0, B->setup>>>(lv.ngroups, (int32_t)lv.tlen, nt, lv.npad,
                                                                    static_cast<const float*>(lv.SLi),
                                                                    static_cast<const float*>(lv.SUi), sl.tiles);
            hs::count_launch();
            if ((e = cudaGetLastError()) != cudaSuccess) rc = hs::cuda_error(e, "batch_tiles_kernel");
        }
    }
    // Every failure from here on releases what the slot holds (in stream
    // order on the setup stream, after the work already queued there).
    auto fail = [&](int code) {
        cudaStreamSynchronize(B->setup);
        if (sl.vec) cudaFreeAsync(sl.vec, B->setup);
        if (sl.tiles) cudaFreeAsync(sl.tiles, B->setup);
        if (sl.soff) cudaFreeAsync(sl.soff, B->setup);
        if (sl.scol) cudaFreeAsync(sl.scol, B->setup);
        if (sl.sval) cudaFreeAsync(sl.sval, B->setup);
        if (sl.P) hs::l1gs_destroy_async(sl.P, B->setup);
        if (sl.A) hs::matrix_destroy_async(sl.A, B->setup);
        return code;
    };
    if (rc) return fail(rc);
    sl.bytes = est;
    const int32_t n = A->n;
    double* x = sl.vec;
    double* r = x + n;
    double* z = r + n;
    double* p = z + n;
    double* b = p + 2 * (size_t)n;
    cudaStream_t st = B->setup;
    cudaError_t ce = cudaMemcpyAsync(b, b_host, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) return fail(hs::cuda_error(ce, "hs_batch_submit: copy of b"));
    const int g = (int)std::min<int64_t>((n + kT - 1) / kT, hsdev::kRedMaxBlocks);
    init_vectors<<<g, kT, 0, st>>>(n, b, x, r);
    hs::count_launch();
    if ((rc = hs_l1gs_apply(sl.P, r, z, HS_F64, st))) return fail(rc);
    init_p_partials<<<g, kT, 0, st>>>(n, z, p, r, b, B->d_init, B->d_init + 2 * hsdev::kRedMaxBlocks);
    init_scalars<<<1, kT, 0, st>>>(B->d_init, B->d_init + 2 * hsdev::kRedMaxBlocks, g, B->d_scal + free_idx,
                                   B->cfg.rtol);
    hs::count_launch(2);
    if ((ce = cudaGetLastError()) != cudaSuccess) return fail(hs::cuda_error(ce, "hs_batch_submit: setup kernels"));
    // No host wait: the next launch orders the solve stream after this
    // admission's setup work through the event.
    if ((ce = cudaEventRecord(B->admitted, st)) != cudaSuccess)
        return fail(hs::cuda_error(ce, "hs_batch_submit: cudaEventRecord"));
    B->pending_admission = true;
    sl.state = 1;
    B->slots[free_idx] = sl;
    B->used += est;
    B->dirty = true;
    if (slot_out) *slot_out = free_idx;
    return HS_OK;
}

int hs_batch_launch(hs_batch* B, int32_t iters) {
    if (!B || iters < 1) return hs::set_error(HS_ERR_ARG, "hs_batch_launch: bad argument");
    if (B->inflight) return hs::set_error(HS_ERR_ARG, "hs_batch_launch: the previous launch was not waited for");
    int rc;
    if (B->pending_admission) {
        HS_CUDA(cudaStreamWaitEvent(B->solve, B->admitted, 0));
        B->pending_admission = false;
    }
    if (B->dirty && (rc = rebuild(B))) return rc;
    if (B->nactive > 0 && B->cfg.schedule == HS_BATCH_PERSISTENT) {
        // one persistent launch for all `iters` iterations, captured once per
        // active set and iteration count
        if (!B->exec || B->exec_iters != iters) {
            if (B->exec) cudaGraphExecDestroy(B->exec);
            if (B->graph) cudaGraphDestroy(B->graph);
            B->exec = nullptr;
            B->graph = nullptr;
            if ((rc = prepare_persistent(B))) return rc;
            cudaStream_t st = B->solve;
            HS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            rc = enqueue_persistent(B, iters, st);
            cudaError_t ce = cudaStreamEndCapture(st, &B->graph);
            if (rc) return rc;
            HS_CUDA(ce);
            HS_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
            B->exec_iters = iters;
        }
        HS_CUDA(cudaGraphLaunch(B->exec, B->solve));
        B->iterations_run += iters;
    } else if (B->nactive > 0) {
        if (!B->exec) {
            // warm launch (kernel attributes), then capture one iteration
            cudaStream_t st = B->solve;
            if ((rc = enqueue_iteration(B, st))) return rc;
            HS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            rc = enqueue_iteration(B, st);
            cudaError_t ce = cudaStreamEndCapture(st, &B->graph);
            if (rc) return rc;
            HS_CUDA(ce);
            HS_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
            B->iterations_run += 1;
            iters -= 1;
        }
        for (int k = 0; k < iters; ++k) HS_CUDA(cudaGraphLaunch(B->exec, B->solve));
        B->iterations_run += iters;
    }
    // Slots admitted while this launch runs are not part of it: their entries
    // in the scalars copy below are not theirs yet.
    for (auto& sl : B->slots) sl.launched = sl.state == 1;
    HS_CUDA(cudaMemcpyAsync(B->h_scal, B->d_scal, sizeof(Scalars) * B->slots.size(), cudaMemcpyDeviceToHost,
                            B->solve));
    HS_CUDA(cudaMemcpyAsync(B->h_ctl, B->d_ctl + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, B->solve));
    HS_CUDA(cudaEventRecord(B->launched, B->solve));
    B->inflight = true;
    return HS_OK;
}

int hs_batch_wait(hs_batch* B, int32_t* finished) {
    if (!B) return hs::set_error(HS_ERR_ARG, "hs_batch_wait: NULL argument");
    int32_t nf = 0;
    if (B->inflight) {
        B->inflight = false;
        HS_CUDA(cudaEventSynchronize(B->launched));
        if (B->h_ctl[0]) {   // a bounded wait of the persistent launch ran out
            B->h_ctl[0] = 0;
            HS_CUDA(cudaMemsetAsync(B->d_ctl + 2, 0, sizeof(int32_t), B->solve));
            HS_CUDA(cudaStreamSynchronize(B->solve));
            B->dirty = true;
            return hs::set_error(HS_ERR_TIMEOUT,
                                 "batched launch: a device-side wait ran out; the active systems' iterates are undefined");
        }
        for (size_t s = 0; s < B->slots.size(); ++s) {
            hs_batch_slot& sl = B->slots[s];
            if (sl.state == 1 && sl.launched && B->h_scal[s].done) {
                sl.state = 2;
                B->dirty = true;
                // the solve stream has passed the event: x is final
                HS_CUDA(cudaMemcpy(sl.x_out, sl.vec, sizeof(double) * sl.n, cudaMemcpyDeviceToHost));
                ++nf;
            }
        }
    }
    if (finished) *finished = nf;
    return HS_OK;
}

int hs_batch_step(hs_batch* B, int32_t iters, int32_t* finished) {
    const int rc = hs_batch_launch(B, iters);
    if (rc) return rc;
    return hs_batch_wait(B, finished);
}

int hs_batch_poll(hs_batch* B, hs_batch_result* results, int32_t max_results, int32_t* count) {
    if (!B || !count || (max_results > 0 && !results)) return hs::set_error(HS_ERR_ARG, "hs_batch_poll: bad argument");
    int32_t c = 0;
    for (size_t s = 0; s < B->slots.size() && c < max_results; ++s) {
        hs_batch_slot& sl = B->slots[s];
        if (sl.state != 2) continue;
        const Scalars& sc = B->h_scal[s];
        results[c].tag = sl.tag;
        results[c].iterations = sc.conv_it;
        results[c].converged = sc.done == 1;
        results[c].relres = sc.bb > 0 ? std::sqrt(sc.rr / sc.bb) : 0.0;
        ++c;
        free_slot(B, sl);
    }
    *count = c;
    return HS_OK;
}

int hs_batch_info_get(const hs_batch* B, hs_batch_info* info) {
    if (!B || !info) return hs::set_error(HS_ERR_ARG, "hs_batch_info_get: NULL argument");
    int32_t a = 0, f = 0;
    for (const auto& s : B->slots) {
        a += s.state == 1;
        f += s.state == 2;
    }
    info->active = a;
    info->finished = f;
    info->hbm_used = B->used;
    info->hbm_budget = B->cfg.hbm_budget;
    info->iterations_run = B->iterations_run;
    return HS_OK;
}

int hs_batch_destroy(hs_batch* B) {
    if (!B) return HS_OK;
    cudaDeviceSynchronize();   // launches and admissions in flight
    for (auto& s : B->slots)
        if (s.state) free_slot(B, s);
    cudaStreamSynchronize(B->solve);   // the stream-ordered frees above
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    void* ptrs[] = {B->d_slots, B->d_scal, B->d_map, B->d_active, B->d_items, B->d_partials, B->d_rzpart,
                    B->d_init, B->d_work, B->d_ctl};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (B->solve) cudaStreamDestroy(B->solve);
    if (B->setup) cudaStreamDestroy(B->setup);
    if (B->launched) cudaEventDestroy(B->launched);
    if (B->admitted) cudaEventDestroy(B->admitted);
    if (B->h_scal) cudaFreeHost(B->h_scal);
    if (B->h_ctl) cudaFreeHost(B->h_ctl);
    delete B;
    return HS_OK;
}

}  // extern "C"
