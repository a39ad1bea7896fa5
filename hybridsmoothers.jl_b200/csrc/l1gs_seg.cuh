// Matrix-view L1 Gauss-Seidel sweep over per-group segment lists.
//
// Reference: the MatrixViewCache sweep of src/l1_gauss_seidel.jl
// (:1588-1597, :1600-1737) scans row i of the (adapted, device-resident)
// matrix on every apply and sums the entries with start <= j < i (forward) or
// i < j <= end (backward) in storage order -- ascending column.  Those
// entries never change, so here they are gathered once, at build time, into
// one stream per group of 32 partitions (lane = partition, as in the packed
// sweeps): for each row of the partitions, in the order the sweep reaches
// them, a number of slots equal to the largest count of any of the 32
// partitions' rows there; slot k of row li holds, for every lane, the value
// and the local column (j - start) of that partition's k-th in-block entry
// ([value x 32][column x 32] per slot, padded to 16 bytes).  A lane's slots past its own count
// hold the value 0 and the column `ps`, a row of y that is always +0: adding
// 0 * 0 leaves an accumulator unchanged bit for bit (an accumulator that
// starts at +0 is never -0), so every lane runs the same slots without a
// count.  Each lane adds its row's entries in storage order with separately
// rounded multiply and add -- the reference's sequence, so results are
// bit-identical.  The apply streams exactly these slots (no out-of-block
// entry, no row pointer) through a per-warp ring filled by 1D bulk copies;
// the per-row slot counts of a group arrive in one 4-byte load per lane and
// are read back by shuffles, and the slot offsets are running sums, so the
// row loop touches no global memory.
#pragma once

#include <stdint.h>

#include "hs_common.cuh"

namespace hsseg {

constexpr int kMaxPartsize = 512;   // y and D_Dl1 of a group in shared memory

// Bytes of a slot of G partitions: [G values][G uint16 columns], padded to 16
// bytes so every slot, and every chunk of slots, is a legal 1D bulk copy.
__host__ __device__ constexpr uint32_t slot_bytes(int G, size_t es) {
    return (uint32_t)((G * (es + 2) + 15) / 16 * 16);
}

// Partitions per group (and per warp): the largest of 32, 16, 8, 4 whose y
// and D_Dl1 slices ((2 ps + 1) rows of G + 1 values) take at most 24 KiB, so
// several warps stay resident per SM.
inline int pick_group(int ps, size_t es) {
    int G = 32;
    while (G > 4 && (size_t)(2 * ps + 1) * (G + 1) * es > 24 * 1024) G /= 2;
    return G;
}

// Device arrays of a segment-list view (one direction).
struct Dir {
    unsigned char* stream = nullptr;   // slots: [value x 32][uint16 column x 32]
    int64_t* base = nullptr;           // first slot of each group
    int32_t* total = nullptr;          // slots of each group
    uint8_t* maxc = nullptr;           // [group][row], row stride ps rounded up to 4: slots of the row
    int64_t slots = 0;                 // all groups
};

struct View {
    Dir lo, up;
    int32_t G = 32;        // partitions per group (lanes that carry a partition)
    int32_t ngroups = 0;
    int64_t bytes = 0;   // device memory held
};

// Builds the lists from a device CSR (row-wise arrays of the preconditioner's
// rows) in smoother type TS; sizes in P's geometry.  Allocates with
// cudaMalloc (accounted in view->bytes).
template <typename TM, typename TS>
int build(int32_t n, int32_t ps, int32_t nparts, const int32_t* rp, const int32_t* ci, const TM* v, bool lower,
          bool upper, View* view, cudaStream_t st);
void destroy(View* view);

struct Params {
    int32_t n, ps, gbeg, gend;
    Dir lo, up;
    const void* D;
    const void* x;
    void* y;
    int32_t* err;
    int32_t vec_io;   // x, y and D_Dl1 are 16-byte aligned
    int32_t G;        // partitions per group
    uint32_t warp_bytes, ring_off, bars_off, tab_off, ys_off, ds_off, mx_off, nst;
};

int launch(int sdt, int io, int sweep, const View& view, int32_t n, int32_t ps, int32_t gbeg, int32_t gend,
           const void* D, const void* x, void* y, int32_t* err, cudaStream_t st);

}  // namespace hsseg
