// One warp's stream of segment-list chunks (l1gs_seg.cuh): the warp's
// (group, direction) pairs in sweep order, each pair's slots copied in chunks
// of K slots into a ring of nst stages by 1D bulk copies (cp.async.bulk, no
// multicast) issued by lane 0, nst chunks ahead of the consumer; waits are
// bounded.  Used by the segment-list apply kernels (l1gs_seg.cu).
#pragma once

#include "l1gs_seg.cuh"

namespace hsseg {

constexpr int kTab = 32;   // (group, direction) pairs whose stream position a warp keeps in shared memory

struct TabEnt {
    int64_t base;   // first slot
    int32_t tot;    // slots
    int32_t pad;
};

// SB: bytes per slot; K: slots per chunk; NDIR: directions per group;
// SWEEP: 0 forward, 1 backward, 2 symmetric.
template <uint32_t SB, int K, int NDIR, int SWEEP>
struct SegStream {
    static constexpr uint32_t CHB = K * SB;   // bytes per chunk
    unsigned char* ring;
    uint64_t* bars;
    TabEnt* tab;
    uint32_t nst;
    int32_t q0, qstride, npairs, total;
    Dir lo, up;
    // producer (lane 0)
    int32_t issued, ppi, pc, pnch, ptot;
    const unsigned char* psrc;
    // consumer
    int32_t ready, freed;

    __device__ __forceinline__ const Dir& dir(int d) const { return (SWEEP == 1 || d == 1) ? up : lo; }

    // Fills the table, counts the warp's chunks, initialises the barriers and
    // issues the first nst chunks.  Called by the whole warp.
    __device__ __forceinline__ void init(int lane, int32_t my_groups) {
        npairs = my_groups * NDIR;
        int32_t nch_lane = 0;
        for (int32_t pi = lane; pi < npairs; pi += 32) {
            const int64_t g = q0 + (int64_t)(pi / NDIR) * qstride;
            const Dir& dd = dir(pi % NDIR);
            const int32_t tot = dd.total[g];
            if (pi < kTab) {
                tab[pi].base = dd.base[g];
                tab[pi].tot = tot;
            }
            nch_lane += (tot + K - 1) / K;
        }
        total = (int32_t)__reduce_add_sync(0xffffffffu, (unsigned)nch_lane);
        issued = 0;
        ppi = 0;
        pc = 0;
        pnch = -1;
        ptot = 0;
        psrc = nullptr;
        ready = 0;
        freed = 0;
        __syncwarp();
        if (lane == 0) {
            for (uint32_t s = 0; s < nst; ++s) hsdev::mbar_init(bars + s, 1);
            hsdev::fence_barrier_init();
            while (issued < total && issued < (int32_t)nst) issue_next();
        }
        __syncwarp();
    }

    // Producer: position on the next chunk; false at the end.
    __device__ __forceinline__ bool advance() {
        while (ppi < npairs) {
            if (pnch < 0) {
                const Dir& dd = dir(ppi % NDIR);
                int64_t b;
                if (ppi < kTab) {
                    b = tab[ppi].base;
                    ptot = tab[ppi].tot;
                } else {
                    const int64_t g = q0 + (int64_t)(ppi / NDIR) * qstride;
                    b = dd.base[g];
                    ptot = dd.total[g];
                }
                pnch = (ptot + K - 1) / K;
                psrc = dd.stream + b * SB;
                pc = 0;
            }
            if (pc < pnch) return true;
            pnch = -1;
            ++ppi;
        }
        return false;
    }

    __device__ __forceinline__ void issue_next() {
        if (!advance()) return;
        const uint32_t s = (uint32_t)issued & (nst - 1u);
        const uint32_t bytes = (uint32_t)min(K, ptot - pc * K) * SB;
        hsdev::mbar_arrive_expect_tx(bars + s, bytes);
        hsdev::bulk_load(ring + (size_t)s * CHB, psrc + (size_t)pc * CHB, bytes, bars + s);
        ++issued;
        ++pc;
    }

    // Bounded wait until chunk `last` has landed (whole warp).
    __device__ __forceinline__ bool wait_upto(int32_t last) {
        while (ready <= last) {
            const bool got =
                hsdev::mbar_wait_bounded(bars + ((uint32_t)ready & (nst - 1u)), ((uint32_t)ready / nst) & 1u);
            if (!__all_sync(0xffffffffu, got)) return false;
            ++ready;
        }
        return true;
    }

    // Chunks below `upto` are consumed: lane 0 refills their stages (whole warp).
    __device__ __forceinline__ void release(int32_t upto, int lane) {
        freed = upto;
        __syncwarp();
        if (lane == 0) {
            hsdev::fence_proxy_async_smem();
            while (issued < total && issued < freed + (int32_t)nst) issue_next();
        }
    }

    __device__ __forceinline__ const unsigned char* slot(int32_t ch, int wi) const {
        return ring + (size_t)((uint32_t)ch & (nst - 1u)) * CHB + (size_t)wi * SB;
    }

    // After a bounded wait ran out: let the copies in flight land (bounded).
    __device__ __forceinline__ void drain() {
        const int32_t end = __shfl_sync(0xffffffffu, issued, 0);
        for (int32_t c = ready; c < end; ++c)
            (void)hsdev::mbar_wait_bounded(bars + ((uint32_t)c & (nst - 1u)), ((uint32_t)c / nst) & 1u);
    }
};

}  // namespace hsseg
